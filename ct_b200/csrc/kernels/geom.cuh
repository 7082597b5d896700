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

// Detector row coordinate of a voxel, vi = H/2 - (zw + h) U (:1008, :1014),
// as a line in the box voxel index z: vi(z) = fma(z, mdv, c0) with
// zw = (z - zPre) vs, mdv = -vs U and c0 = H/2 - (h - zPre vs) U. One fused
// multiply-add per voxel; the backprojectors and the forward projector all use
// exactly this form so that they take the same row decisions.
struct RowLine {
    float mdv, c0;
};

__device__ __forceinline__ RowLine row_line(float U, float h, float zpv, float vs, float vPre) {
    RowLine r;
    r.mdv = -__fmul_rn(vs, U);
    r.c0 = fmaf(-__fsub_rn(h, zpv), U, vPre);
    return r;
}

__device__ __forceinline__ float row_at(const RowLine& r, float zf) { return fmaf(zf, r.mdv, r.c0); }

// A row coordinate is inside the detector when 0 <= vi <= H - 1.1
// (the v bounds of :927-928 and :1011 expressed on vi).
__device__ __forceinline__ bool row_ok(float vi, float vi_hi) { return vi >= 0.0f && vi <= vi_hi; }

}  // namespace ctb
