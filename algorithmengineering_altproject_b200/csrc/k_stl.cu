// Surface export of a design (io.cpp:80-87): boundary faces of the voxels with density >= iso
// (voxel_surface.hpp:12-93), written as the records of a binary STL (export_stl.hpp:14-33), in the
// reference's order so that the file is byte-identical.
//
// The reference visits voxels in full-index order k = y + ny*x + ny*nx*z (y is the grid row, fea.cpp:222)
// and per inside voxel emits the faces -X, +X, -Y, +Y, -Z, +Z whose neighbour is outside or absent, each
// as 2 triangles.  On the device: (1) each block counts the faces of a chunk of consecutive k,
// (2) one block scans the chunk totals, (3) each block recounts its chunk, scans the per-thread counts
// and writes its 50-byte records (zero normal, 3 vertices, zero attribute) at their final offsets.
#include "kernels.hpp"

namespace t3d {

namespace {

constexpr int STL_THREADS = 256, STL_ITEMS = 16, STL_CHUNK = STL_THREADS * STL_ITEMS;

// bit f set when face f (-X, +X, -Y, +Y, -Z, +Z) of voxel (x, y, z) is on the surface
__device__ __forceinline__ int face_bits(const Grid& g, const float* __restrict__ d, float iso, int x, int y, int z) {
    auto in = [&](int xx, int yy, int zz) { return d[g.cell(xx, yy, zz)] >= iso; };
    if (!in(x, y, z)) return 0;
    int b = 0;
    if (x == 0 || !in(x - 1, y, z)) b |= 1;
    if (x == g.nx - 1 || !in(x + 1, y, z)) b |= 2;
    if (y == 0 || !in(x, y - 1, z)) b |= 4;
    if (y == g.ny - 1 || !in(x, y + 1, z)) b |= 8;
    if (z == 0 || !in(x, y, z - 1)) b |= 16;
    if (z == g.nz - 1 || !in(x, y, z + 1)) b |= 32;
    return b;
}

__device__ __forceinline__ int voxel_faces(const Grid& g, const float* d, float iso, int64_t k) {
    const int y = (int)(k % g.ny);
    const int64_t r = k / g.ny;
    const int x = (int)(r % g.nx), z = (int)(r / g.nx);
    return face_bits(g, d, iso, x, y, z);
}

// exclusive scan of one value per thread over the block; *total = block sum
__device__ __forceinline__ unsigned block_exclusive_scan(unsigned v, unsigned* sh, unsigned* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) sh[w] = inc;
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        unsigned s = lane < nw ? sh[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned t = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += t;
        }
        if (lane < nw) sh[lane] = s;   // inclusive warp totals
    }
    __syncthreads();
    const unsigned before = (w > 0 ? sh[w - 1] : 0u) + inc - v;
    *total = sh[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before;
}

__global__ void __launch_bounds__(STL_THREADS) k_stl_count(Grid g, const float* __restrict__ d, float iso,
                                                           unsigned* __restrict__ bsum) {
    __shared__ unsigned sh[32];
    const int64_t nv = (int64_t)g.nx * g.ny * g.nz;
    const int64_t base = (int64_t)blockIdx.x * STL_CHUNK + (int64_t)threadIdx.x * STL_ITEMS;
    unsigned c = 0;
    for (int i = 0; i < STL_ITEMS; ++i)
        if (base + i < nv) c += __popc(voxel_faces(g, d, iso, base + i));
    unsigned total;
    block_exclusive_scan(c, sh, &total);
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// exclusive scan of the nb chunk totals (one block); bsum[nb] = total faces
__global__ void __launch_bounds__(1024) k_stl_scan(unsigned* __restrict__ bsum, int nb) {
    __shared__ unsigned sh[32];
    unsigned carry = 0;
    for (int b0 = 0; b0 < nb; b0 += blockDim.x) {
        const int i = b0 + threadIdx.x;
        const unsigned v = i < nb ? bsum[i] : 0u;
        unsigned total;
        const unsigned ex = block_exclusive_scan(v, sh, &total);
        if (i < nb) bsum[i] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) bsum[nb] = carry;
}

__device__ __forceinline__ void put_f(uint16_t* p, float v) {
    const unsigned b = __float_as_uint(v);
    p[0] = (uint16_t)(b & 0xffffu);
    p[1] = (uint16_t)(b >> 16);
}

// the 2 triangles of one face (voxel_surface.hpp:17-43) as STL records at record index t
__device__ void write_face(uint16_t* __restrict__ body, int64_t t, int axis, float x0, float y0, float z0) {
    float v[4][3];
#pragma unroll
    for (int i = 0; i < 4; ++i) { v[i][0] = x0; v[i][1] = y0; v[i][2] = z0; }
    if (axis == 0) {          // plane x = const: vary y, z
        v[1][1] += 1.0f; v[2][1] += 1.0f; v[2][2] += 1.0f; v[3][2] += 1.0f;
    } else if (axis == 1) {   // plane y = const: vary x, z
        v[1][0] += 1.0f; v[2][0] += 1.0f; v[2][2] += 1.0f; v[3][2] += 1.0f;
    } else {                  // plane z = const: vary x, y
        v[1][0] += 1.0f; v[2][0] += 1.0f; v[2][1] += 1.0f; v[3][1] += 1.0f;
    }
    const int tri[2][3] = {{0, 1, 2}, {0, 2, 3}};
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        uint16_t* r = body + 25 * (t + s);
#pragma unroll
        for (int i = 0; i < 6; ++i) r[i] = 0;            // normal (0, 0, 0)
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int c = 0; c < 3; ++c) put_f(r + 6 + 6 * k + 2 * c, v[tri[s][k]][c]);
        r[24] = 0;                                        // attribute
    }
}

__global__ void __launch_bounds__(STL_THREADS) k_stl_write(Grid g, const float* __restrict__ d, float iso,
                                                           const unsigned* __restrict__ boff,
                                                           uint16_t* __restrict__ body) {
    __shared__ unsigned sh[32];
    const int64_t nv = (int64_t)g.nx * g.ny * g.nz;
    const int64_t base = (int64_t)blockIdx.x * STL_CHUNK + (int64_t)threadIdx.x * STL_ITEMS;
    unsigned c = 0;
    for (int i = 0; i < STL_ITEMS; ++i)
        if (base + i < nv) c += __popc(voxel_faces(g, d, iso, base + i));
    unsigned total;
    int64_t face = (int64_t)boff[blockIdx.x] + block_exclusive_scan(c, sh, &total);
    for (int i = 0; i < STL_ITEMS; ++i) {
        const int64_t k = base + i;
        if (k >= nv) break;
        const int y = (int)(k % g.ny);
        const int64_t r = k / g.ny;
        const int x = (int)(r % g.nx), z = (int)(r / g.nx);
        const int b = face_bits(g, d, iso, x, y, z);
        if (!b) continue;
        const float fx = (float)x, fy = (float)y, fz = (float)z;
        if (b & 1) { write_face(body, 2 * face, 0, fx, fy, fz); ++face; }
        if (b & 2) { write_face(body, 2 * face, 0, fx + 1.0f, fy, fz); ++face; }
        if (b & 4) { write_face(body, 2 * face, 1, fx, fy, fz); ++face; }
        if (b & 8) { write_face(body, 2 * face, 1, fx, fy + 1.0f, fz); ++face; }
        if (b & 16) { write_face(body, 2 * face, 2, fx, fy, fz); ++face; }
        if (b & 32) { write_face(body, 2 * face, 2, fx, fy, fz + 1.0f); ++face; }
    }
}

}  // namespace

int stl_chunks(const Grid& g) {
    const int64_t nv = (int64_t)g.nx * g.ny * g.nz;
    return (int)((nv + STL_CHUNK - 1) / STL_CHUNK);
}

void launch_stl_count(const Grid& g, const float* d, float iso, unsigned* bsum, cudaStream_t s) {
    const int nb = stl_chunks(g);
    k_stl_count<<<nb, STL_THREADS, 0, s>>>(g, d, iso, bsum);
    k_stl_scan<<<1, 1024, 0, s>>>(bsum, nb);
}

void launch_stl_write(const Grid& g, const float* d, float iso, const unsigned* boff, uint16_t* body, cudaStream_t s) {
    k_stl_write<<<stl_chunks(g), STL_THREADS, 0, s>>>(g, d, iso, boff, body);
}

}  // namespace t3d
