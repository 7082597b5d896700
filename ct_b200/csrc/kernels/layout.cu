// Output layout kernel: X-fastest device slab -> requested index order and
// byte order. Replaces the per-voxel QDataStream walk of
// Volume<float>::saveToBinaryFile (Common/Volume.h:476-574): same-layout
// writes are linear; Z_FASTEST output walks x -> y -> z (idx = x*Y*Z + y*Z + z).
// Here the transpose runs through 32x32 shared-memory tiles so that both the
// read (along x) and the write (along z) are coalesced; big-endian output
// swaps the four bytes of each float on the way.

#include "../ctb_internal.h"

namespace ctb {

namespace {

__device__ __forceinline__ uint32_t maybe_swap(float v, int swap) {
    const uint32_t b = __float_as_uint(v);
    return swap ? __byte_perm(b, 0, 0x0123) : b;
}

// in: [zs][y][x]  ->  out: [x][y][zs]
__global__ void zfastest_kernel(const float* __restrict__ in, int X, int Y, int Zs, int swap,
                                uint32_t* __restrict__ out) {
    __shared__ float tile[32][33];
    const int xt = blockIdx.x * 32, zt = blockIdx.y * 32, y = blockIdx.z;
    const long long plane = (long long)X * Y;
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int z = zt + j, x = xt + threadIdx.x;
        if (z < Zs && x < X) tile[j][threadIdx.x] = in[(long long)z * plane + (long long)y * X + x];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int x = xt + j, z = zt + threadIdx.x;
        if (z < Zs && x < X) out[((long long)x * Y + y) * Zs + z] = maybe_swap(tile[threadIdx.x][j], swap);
    }
}

__global__ void swap_kernel(const float* __restrict__ in, long long n, uint32_t* __restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = maybe_swap(in[i], 1);
}

}  // namespace

int layout_launch(const float* src, int x, int y, int zs, int index_order, int byte_order, void* dst,
                  cudaStream_t s) {
    if (x <= 0 || y <= 0 || zs <= 0) return CTB_OK;
    const int swap = byte_order == CTB_BIG_ENDIAN;
    if (index_order == CTB_Z_FASTEST) {
        if (y > 65535) { set_global_error("layout: y too large"); return CTB_ERR_UNSUPPORTED; }
        dim3 grid((x + 31) / 32, (zs + 31) / 32, y);
        zfastest_kernel<<<grid, dim3(32, 8), 0, s>>>(src, x, y, zs, swap, (uint32_t*)dst);
    } else if (swap) {
        const long long n = (long long)x * y * zs;
        swap_kernel<<<148 * 8, 256, 0, s>>>(src, n, (uint32_t*)dst);
    } else {
        CTB_CUDA_TRY(cudaMemcpyAsync(dst, src, sizeof(float) * (size_t)x * y * zs, cudaMemcpyDeviceToDevice, s));
    }
    return cuda_status(cudaGetLastError(), "layout kernel launch");
}

}  // namespace ctb
