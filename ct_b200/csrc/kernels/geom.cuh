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

// Bounds-checked build (-DCTB_BOUNDS_CHECK, libctb_checked.so): every texel
// fetch of the backprojectors is checked against the buffer it reads (the
// staged box, or the projections in global memory) before it is made. A
// fetch out of range is skipped (reads as 0) and recorded in this file's
// status words: a count and the first offender (site << 56 | index). Nothing
// traps. In the normal build the checks compile to nothing.
#ifdef CTB_BOUNDS_CHECK
static __device__ unsigned int g_bounds_count;
static __device__ unsigned long long g_bounds_first;
__device__ __forceinline__ bool fetch_ok(long long idx, long long lim, unsigned site) {
    if (idx >= 0 && idx < lim) return true;
    atomicAdd(&g_bounds_count, 1u);
    atomicCAS(&g_bounds_first, 0ull,
              (static_cast<unsigned long long>(site) << 56) | (static_cast<unsigned long long>(idx) & ((1ull << 56) - 1)));
    return false;
}
#define CTB_FETCH_OK(idx, lim, site) ::ctb::fetch_ok((idx), (lim), (site))
#else
#define CTB_FETCH_OK(idx, lim, site) true
#endif

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
// as a line in the box voxel index z: vi(z) = z mdv + c0 with zw = (z - zPre)
// vs, mdv = -vs U and c0 = H/2 - (h - zPre vs) U, evaluated from the start of
// z's block of 32 slices:
//     vi(z) = fma(z mod 32, mdv, fma(z - z mod 32, mdv, c0)).
// Every path (the backprojectors' pair loop and per-voxel loops, the gather
// backprojector, the forward projector) forms rows this way, so they take the
// same row decisions for any slab or tile split. The block origin lets the
// shared-memory backprojector's pair loop, whose tiles of 32 slices start on
// a block, take z mod 32 as an immediate operand with one row origin per
// view, instead of holding 32 slice coordinates in registers (the freed
// registers let the compiler overlap voxel pairs: 6 % faster for FP16).
struct RowLine {
    float mdv, c0;
};

__device__ __forceinline__ RowLine row_line(float U, float h, float zpv, float vs, float vPre) {
    RowLine r;
    r.mdv = -__fmul_rn(vs, U);
    r.c0 = fmaf(-__fsub_rn(h, zpv), U, vPre);
    return r;
}

// row origin of the block of 32 slices that starts at box slice zb (a multiple of 32)
__device__ __forceinline__ float row_block(const RowLine& r, int zb) { return fmaf(float(zb), r.mdv, r.c0); }

// row of box slice z (z >= 0)
__device__ __forceinline__ float row_at(const RowLine& r, int z) {
    const int zo = z & 31;
    return fmaf(float(zo), r.mdv, row_block(r, z - zo));
}

// Whether a voxel falls inside the detector's rows, decided exactly as the
// reference decides it (:926-928, :1008-1011): v = (z + h) U rounded in float
// and kept when lbV <= v <= ubV, with zw the voxel's world z. The row line
// above gives the row and its weight; near the first and last row its
// rounding can land on the other side of a bound that the reference's v hits
// exactly (a voxel whose v equals ubV, row 0), so membership is taken from
// here. A kept voxel's row line value then lies within rounding of [0, H-1.1],
// and int() of it still names rows inside the detector.
__device__ __forceinline__ bool v_inside(float zw, float h, float U, float lbV, float ubV) {
    const float v = __fmul_rn(__fadd_rn(zw, h), U);
    return v >= lbV && v <= ubV;
}

// The same decision for the n slices zs .. zs+n-1 of one column at once: v
// grows with z (U > 0, vs > 0) and rounding keeps it monotone, so the kept
// slices are one run [*ja, *jb] (local indices; empty when *ja > *jb). Its
// ends are estimated from the continuous v and settled with v_inside's own
// arithmetic (a step or two), instead of testing every slice.
__device__ __forceinline__ void v_inside_run(int zs, int n, float zPre, float vs, float h, float U, float lbV,
                                             float ubV, int* ja, int* jb) {
    auto v = [&](int j) { return __fmul_rn(__fadd_rn(__fmul_rn(__fsub_rn(float(zs + j), zPre), vs), h), U); };
    const float rv = 1.0f / vs, ru = 1.0f / U, base = zPre - float(zs);
    // last j with v <= ubV
    int b = int(floorf(fminf(fmaxf((ubV * ru - h) * rv + base, -1.0f), float(n - 1))));
    while (b + 1 <= n - 1 && v(b + 1) <= ubV) ++b;
    while (b >= 0 && v(b) > ubV) --b;
    // first j with v >= lbV
    int a = int(ceilf(fminf(fmaxf((lbV * ru - h) * rv + base, 0.0f), float(n))));
    while (a - 1 >= 0 && v(a - 1) >= lbV) --a;
    while (a <= n - 1 && v(a) < lbV) ++a;
    *ja = a;
    *jb = b;
}

}  // namespace ctb
