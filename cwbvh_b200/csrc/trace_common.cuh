// Device-side building blocks shared by the CWBVH and BVH2 trace kernels.
//
// Arithmetic contract.  Every floating-point step of the slab and triangle
// tests is written with explicit round-to-nearest intrinsics (__fmaf_rn,
// __fmul_rn, __fsub_rn, __frcp_rn), so the compiler cannot re-associate or
// re-contract them and the CPU oracle reproduces them bit for bit with fmaf()
// and IEEE division.  The expressions follow the reference's source order with
// products folded into fused multiply-adds the way a*b+c contracts
// (src/TraversalKernelCWBVH.cu:134-139,166-202,322-332;
// src/TraversalKernelBVH2.cu:14-24,135-149).  One deliberate difference: the
// reference is built with -use_fast_math (CMakeLists.txt:9), whose 1/x is an
// approximate reciprocal; here 1/x is correctly rounded, which makes results
// reproducible on the CPU and at least as accurate.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "device_api.h"

namespace rq {

constexpr unsigned kFullMask = 0xFFFFFFFFu;
constexpr float kOoeps = 0x1p-80f;           // 2^-80, src/TraversalKernelCWBVH.cu:31

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Read-only (non-coherent) 16-byte load of node and triangle data.
__device__ __forceinline__ float4 ld_nc(const float4* p) { return __ldg(p); }

__device__ __forceinline__ unsigned highest_bit(unsigned x) { return 31u - (unsigned)__clz(x); }

// Min/max of floats compared as signed 32-bit integers, as the reference's
// video-instruction helpers do (src/FastDeviceMinMax.h:44-51).  For
// non-negative values this is the float order; negative values compare in
// reverse, and the result is what the reference computes in either case.
__device__ __forceinline__ float imax3(float a, float b, float c) {
    return __int_as_float(max(max(__float_as_int(a), __float_as_int(b)), __float_as_int(c)));
}
__device__ __forceinline__ float imin3(float a, float b, float c) {
    return __int_as_float(min(min(__float_as_int(a), __float_as_int(b)), __float_as_int(c)));
}
// max(min(a, b), c) and min(max(a, b), c) on integer bits (vmin/vmax with a
// secondary op, src/FastDeviceMinMax.h:45-46).
__device__ __forceinline__ float imin_then_max(float a, float b, float c) {
    return __int_as_float(max(min(__float_as_int(a), __float_as_int(b)), __float_as_int(c)));
}
__device__ __forceinline__ float imax_then_min(float a, float b, float c) {
    return __int_as_float(min(max(__float_as_int(a), __float_as_int(b)), __float_as_int(c)));
}

// 1/d with the 2^-80 guard against division by zero (src/TraversalKernelCWBVH.cu:78-80).
__device__ __forceinline__ float guarded_rcp(float d) {
    return __frcp_rn(fabsf(d) > kOoeps ? d : copysignf(kOoeps, d));
}

// Woop ray-triangle test (src/TraversalKernelCWBVH.cu:318-347).  Returns true
// when tmin < t < tmax, 0 <= u <= 1, v >= 0 and u + v <= 1.
__device__ __forceinline__ bool woop_test(const float4& v0, const float4& v1, const float4& v2, float ox,
                                          float oy, float oz, float dx, float dy, float dz, float tmin,
                                          float tmax, float& t, float& u, float& v) {
    const float Oz = __fmaf_rn(-oz, v0.z, __fmaf_rn(-oy, v0.y, __fmaf_rn(-ox, v0.x, v0.w)));
    const float Dz = __fmaf_rn(dz, v0.z, __fmaf_rn(dx, v0.x, __fmul_rn(dy, v0.y)));
    t = __fmul_rn(Oz, __frcp_rn(Dz));
    const float Ox = __fmaf_rn(oz, v1.z, __fmaf_rn(oy, v1.y, __fmaf_rn(ox, v1.x, v1.w)));
    const float Dx = __fmaf_rn(dz, v1.z, __fmaf_rn(dx, v1.x, __fmul_rn(dy, v1.y)));
    u = __fmaf_rn(t, Dx, Ox);
    const float Oy = __fmaf_rn(oz, v2.z, __fmaf_rn(oy, v2.y, __fmaf_rn(ox, v2.x, v2.w)));
    const float Dy = __fmaf_rn(dz, v2.z, __fmaf_rn(dx, v2.x, __fmul_rn(dy, v2.y)));
    v = __fmaf_rn(t, Dy, Oy);
    return (t > tmin && t < tmax) && (u >= 0.0f && u <= 1.0f) && (v >= 0.0f && __fadd_rn(u, v) <= 1.0f);
}

// Exact float of byte `byte_index` of a word (every byte value is a float),
// two ways that run on different pipes.  The integer conversion of the
// extracted byte takes fewer instructions (the whole trace kernel issues 14 %
// fewer warp instructions per ray than with the permute form alone) but runs
// on the XU pipe; building 2^23 + b with a byte permute and subtracting 2^23
// runs on the ALU and FMA pipes.  The slab test converts the x and y bytes
// the first way and the z bytes the second, which measured 1-3 % faster than
// either way alone.
__device__ __forceinline__ float byte_to_float(unsigned word, unsigned byte_index) {
    return __uint2float_rn((word >> (8u * byte_index)) & 0xFFu);
}
__device__ __forceinline__ float byte_to_float_permute(unsigned word, unsigned byte_index) {
    const unsigned sel = 0x7540u | byte_index;  // bytes: [word.b<i>, 0, 0, 0x4B]
    unsigned r;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(word), "r"(0x4B000000u), "r"(sel));
    return __fsub_rn(__uint_as_float(r), 8388608.0f);
}

// Hit mask of the 8 children of one CWBVH node (src/TraversalKernelCWBVH.cu:
// 141-288): bits 24-31 for inner children at 24 + (slot ^ octinv), the
// unary triangle counts at their offsets for leaf children.  The slab
// extremes are taken as the reference does, on the float bits compared as
// signed integers, then clamped by tmin / tmax with float min/max.
__device__ __forceinline__ unsigned cwbvh_hitmask(const float4& n1, const float4& n2, const float4& n3,
                                                  const float4& n4, float adjx, float adjy, float adjz, float orx,
                                                  float ory, float orz, bool negx, bool negy, bool negz,
                                                  unsigned octinv4, float tmin, float tmax) {
    unsigned hitmask = 0u;
#pragma unroll
    for (int g = 0; g < 2; ++g) {
        const unsigned meta4 = __float_as_uint(g == 0 ? n1.z : n1.w);
        const unsigned inner4 = ((meta4 & (meta4 << 1)) & 0x10101010u) >> 4;
        const unsigned bitidx4 = (meta4 ^ (octinv4 & (inner4 * 0xFFu))) & 0x1F1F1F1Fu;
        const unsigned bits4 = (meta4 >> 5) & 0x07070707u;
        const unsigned wlx = __float_as_uint(g == 0 ? n2.x : n2.y);
        const unsigned whx = __float_as_uint(g == 0 ? n3.z : n3.w);
        const unsigned wly = __float_as_uint(g == 0 ? n2.z : n2.w);
        const unsigned why = __float_as_uint(g == 0 ? n4.x : n4.y);
        const unsigned wlz = __float_as_uint(g == 0 ? n3.x : n3.y);
        const unsigned whz = __float_as_uint(g == 0 ? n4.z : n4.w);
        const unsigned lox = negx ? whx : wlx, hix = negx ? wlx : whx;
        const unsigned loy = negy ? why : wly, hiy = negy ? wly : why;
        const unsigned loz = negz ? whz : wlz, hiz = negz ? wlz : whz;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const float tx0 = __fmaf_rn(byte_to_float(lox, c), adjx, orx);
            const float ty0 = __fmaf_rn(byte_to_float(loy, c), adjy, ory);
            const float tz0 = __fmaf_rn(byte_to_float_permute(loz, c), adjz, orz);
            const float tx1 = __fmaf_rn(byte_to_float(hix, c), adjx, orx);
            const float ty1 = __fmaf_rn(byte_to_float(hiy, c), adjy, ory);
            const float tz1 = __fmaf_rn(byte_to_float_permute(hiz, c), adjz, orz);
            const float cmin = fmaxf(imax3(tx0, ty0, tz0), tmin);
            const float cmax = fminf(imin3(tx1, ty1, tz1), tmax);
            if (cmin <= cmax) hitmask |= ((bits4 >> (8 * c)) & 0xFFu) << ((bitidx4 >> (8 * c)) & 0xFFu);
        }
    }
    return hitmask;
}

}  // namespace rq
