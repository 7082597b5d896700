// Per-column projection geometry shared by the backprojector and the forward
// projector. Every operation is an explicitly rounded IEEE single-precision op
// (no fused multiply-add), in the order of the reference CPU path
// (Ct/CtVolume.cpp:977-996):
//     t = (-1)*x*sin + y*cos; t += uOffset; s = x*cos + y*sin
//     U = D / (D - s);  u = t * U
// so the two projectors take identical discrete decisions (cylinder, bounds,
// u0, v0) and match the reference's float arithmetic.
#pragma once

#include "../ctb_internal.h"

namespace ctb {

__device__ __forceinline__ float world_coord(int idx, float pre, float vs) {
    return __fmul_rn(__fsub_rn(float(idx), pre), vs);
}

__device__ __forceinline__ bool in_cylinder(float xw, float yw, float r2) {
    return __fadd_rn(__fmul_rn(xw, xw), __fmul_rn(yw, yw)) < r2;
}

__device__ __forceinline__ void column_geom(float xw, float yw, float sn, float cs, float D, float uOff, float* U,
                                            float* u) {
    float t = __fadd_rn(__fmul_rn(__fmul_rn(-1.0f, xw), sn), __fmul_rn(yw, cs));
    t = __fadd_rn(t, uOff);
    const float s = __fadd_rn(__fmul_rn(xw, cs), __fmul_rn(yw, sn));
    *U = __fdiv_rn(D, __fsub_rn(D, s));
    *u = __fmul_rn(t, *U);
}

// Detector row coordinate of a voxel: vi = (-1)*((z + h) * U) + H/2 (:1008, :1014).
__device__ __forceinline__ float row_coord(float zw, float h, float U, float vPre, float* v) {
    *v = __fmul_rn(__fadd_rn(zw, h), U);
    return __fadd_rn(-*v, vPre);
}

}  // namespace ctb
