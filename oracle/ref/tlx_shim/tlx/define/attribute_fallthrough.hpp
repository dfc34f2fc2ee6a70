// Project-written stand-in for the tlx header of the same name: the
// fallthrough attribute marker used in switch statements.
#pragma once
#define TLX_ATTRIBUTE_FALLTHROUGH [[gnu::fallthrough]]
