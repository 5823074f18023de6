// TEST INFRASTRUCTURE ONLY (oracle).  The handful of SDL3 names the
// reference's CPU scene headers use, so they compile without SDL: fixed-width
// typedefs and SDL_assert.  Nothing graphical is declared.
#pragma once
#include <cassert>
#include <cstdint>
typedef uint8_t Uint8;
typedef int8_t Sint8;
typedef uint16_t Uint16;
typedef int16_t Sint16;
typedef uint32_t Uint32;
typedef int32_t Sint32;
typedef uint64_t Uint64;
typedef int64_t Sint64;
#define SDL_assert(x) assert(x)
