// Two neurons per thread with packed float32 pairs (sm_100a add/sub/mul .f32x2).
//
// The LIF and AdEx updates under Euler, RK2 and RK4 are chains of elementwise
// float operations, identical for every neuron of a population.  A thread that
// advances two neurons with the packed instructions issues one instruction per
// operation pair, and shares its loop, ballot and parameter overhead between the
// two.  Each packed operation is the IEEE round-to-nearest operation on each
// lane, so a lane's result is bit-for-bit the scalar code's (eb_device.cuh): the
// expressions below keep the scalar operand order.  Anything that branches per
// neuron -- the AdEx regimes above the exponential's cut-off, LIF refractoriness,
// table lookups, spikes, resets -- runs per lane on the scalar code.
#pragma once
#include <cstdint>
#include "eb_device.cuh"

namespace eb {

struct F2 {
    unsigned long long v;  // lane 0 in the low word, lane 1 in the high word
};

__device__ __forceinline__ F2 f2(float a, float b) {
    F2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ F2 f2(float a) { return f2(a, a); }
__device__ __forceinline__ float lane0(F2 x) { return __uint_as_float((unsigned)(x.v & 0xffffffffull)); }
__device__ __forceinline__ float lane1(F2 x) { return __uint_as_float((unsigned)(x.v >> 32)); }
__device__ __forceinline__ float lane(F2 x, int l) { return l == 0 ? lane0(x) : lane1(x); }
__device__ __forceinline__ void set_lane(F2 &x, int l, float v) { x = l == 0 ? f2(v, lane1(x)) : f2(lane0(x), v); }

__device__ __forceinline__ F2 operator+(F2 a, F2 b) {
    F2 r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
__device__ __forceinline__ F2 operator-(F2 a, F2 b) {
    F2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
__device__ __forceinline__ F2 operator*(F2 a, F2 b) {
    F2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}

}  // namespace eb
