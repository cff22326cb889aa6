/* Force-included when compiling the reference's CUDA sources for sm_100a:
 * maps the legacy intrinsic names they use (removed from current CUDA) to
 * their current spellings.  Part of the oracle/_ref build recipe only. */
#pragma once
#define float_as_uint __float_as_uint
#define uint_as_float __uint_as_float
#define int_as_float __int_as_float
