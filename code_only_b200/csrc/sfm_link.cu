// sfm_link.cu -- the block links of an AMR hierarchy built on the device.
//
// After each refinement the reference derives every new block's links from
// its parent's: ParentGid, ChildGid(lri,lrj,lrk) and NeighborGid(lr,dir),
// the neighbours being children of the parent or of the parent's neighbours
// (update_neighbor, update_neighbor_linklist, update_parent_linklist;
// grid.F90:587-731), and fmg_make_linklist copies them into the solver's
// structure (fmg_data_if.F90:298-411).  sfm_link_blocks computes the same
// links from the blocks' levels and integer positions alone, so a hierarchy
// regridded on the device needs no round trip through the host: one hash
// table keyed by (level, i, j, k) in device memory, one lookup per link.
//
//   parent    the block at level L - 1 holding (i/2, j/2, k/2)
//   child c   the block at level L + 1 at (2i + c&1, 2j + (c>>1)&1, 2k + (c>>2)&1)
//   nbr f     f = lr + 2 dir: the block at level L one step left (lr = 0) or
//             right along dir; a periodic direction wraps at the level's
//             extent ngb[dir] << L, another one gives -1 and touch = 1 there
//
// The table is open-addressed (linear probing, twice as many slots as
// blocks, so every probe sequence ends at an empty slot within the table);
// the result does not depend on insertion order.  A duplicated block, a
// block above the base level without a parent, or a block with some but
// not all of its 8 children is reported as SFM_EHIER.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/sfmg.h"

namespace {

constexpr uint64_t kEmpty = ~(uint64_t)0;
constexpr int kCoordBits = 20;   // i, j, k < 2^20 on every level
constexpr int kMaxLevels = 16;   // level < 2^4 above the three coordinates

struct LinkTable {
    uint64_t *keys;
    int32_t *vals;
    uint64_t mask;   // slots - 1 (slots a power of two)
};

__host__ __device__ __forceinline__ uint64_t link_key(int L, int64_t i, int64_t j, int64_t k) {
    return ((uint64_t)L << (3 * kCoordBits)) | ((uint64_t)k << (2 * kCoordBits)) | ((uint64_t)j << kCoordBits) |
           (uint64_t)i;
}
__device__ __forceinline__ uint64_t link_hash(uint64_t x) {   // 64-bit finaliser (murmur3 fmix64)
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return x;
}

__global__ void k_link_clear(LinkTable t) {
    for (uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; s <= t.mask;
         s += (uint64_t)gridDim.x * blockDim.x)
        t.keys[s] = kEmpty;
}

__global__ void k_link_insert(LinkTable t, int nb, int nlev, const int32_t *level, const int32_t *ijk, int3 ngb,
                              int *err) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        const int L = level[b];
        const int64_t i = ijk[3 * b], j = ijk[3 * b + 1], k = ijk[3 * b + 2];
        if (L < 0 || L >= nlev || i < 0 || j < 0 || k < 0 || i >= ((int64_t)ngb.x << L) ||
            j >= ((int64_t)ngb.y << L) || k >= ((int64_t)ngb.z << L)) {   // outside its level's box
            atomicExch(err, 1);
            continue;
        }
        const uint64_t key = link_key(L, i, j, k);
        uint64_t s = link_hash(key) & t.mask;
        for (uint64_t probe = 0; probe <= t.mask; probe++, s = (s + 1) & t.mask) {
            const unsigned long long prev =
                atomicCAS(reinterpret_cast<unsigned long long *>(t.keys + s), (unsigned long long)kEmpty,
                          (unsigned long long)key);
            if (prev == kEmpty) {
                t.vals[s] = b;
                break;
            }
            if (prev == key) {   // the same block twice
                atomicExch(err, 1);
                break;
            }
        }
    }
}

// the block at (L, i, j, k), or -1; the table was filled by a completed launch
__device__ int32_t link_find(const LinkTable &t, int L, int64_t i, int64_t j, int64_t k) {
    const uint64_t key = link_key(L, i, j, k);
    uint64_t s = link_hash(key) & t.mask;
    for (uint64_t probe = 0; probe <= t.mask; probe++, s = (s + 1) & t.mask) {
        const uint64_t v = t.keys[s];
        if (v == key) return t.vals[s];
        if (v == kEmpty) return -1;
    }
    return -1;
}

__global__ void k_link_lookup(LinkTable t, int nb, int nlev, const int32_t *level, const int32_t *ijk, int3 ngb,
                              int3 per, int32_t *parent, int32_t *child, int32_t *nbr, int8_t *touch, int *err) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        const int L = level[b];
        const int64_t q[3] = {ijk[3 * b], ijk[3 * b + 1], ijk[3 * b + 2]};
        if (L < 0 || L >= nlev) continue;   // reported by k_link_insert
        int32_t p = -1;
        if (L > 0) {
            p = link_find(t, L - 1, q[0] >> 1, q[1] >> 1, q[2] >> 1);
            if (p < 0) atomicExch(err, 1);
        }
        parent[b] = p;
        int found = 0;
        for (int c = 0; c < 8; c++) {
            const int32_t cb = L + 1 < nlev
                                   ? link_find(t, L + 1, 2 * q[0] + (c & 1), 2 * q[1] + ((c >> 1) & 1),
                                               2 * q[2] + ((c >> 2) & 1))
                                   : -1;
            child[8 * b + c] = cb;
            found += cb >= 0;
        }
        if (found != 0 && found != 8) atomicExch(err, 1);
        const int64_t ext[3] = {(int64_t)ngb.x << L, (int64_t)ngb.y << L, (int64_t)ngb.z << L};
        const int pd[3] = {per.x, per.y, per.z};
        for (int dir = 0; dir < 3; dir++)
            for (int lr = 0; lr < 2; lr++) {
                int64_t r[3] = {q[0], q[1], q[2]};
                r[dir] += lr == 0 ? -1 : 1;
                const bool out = r[dir] < 0 || r[dir] >= ext[dir];
                int32_t nbb = -1;
                if (out && pd[dir]) r[dir] = (r[dir] + ext[dir]) % ext[dir];
                if (!out || pd[dir]) nbb = link_find(t, L, r[0], r[1], r[2]);
                nbr[6 * b + lr + 2 * dir] = nbb;
                touch[6 * b + lr + 2 * dir] = (int8_t)(out && !pd[dir]);
            }
    }
}

bool on_device(const void *p, int dev) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == dev;
}

}  // namespace

extern "C" int sfm_link_blocks(int32_t nblocks, int32_t nlev, const int32_t *d_level, const int32_t *d_ijk,
                               const int32_t ngb[3], const int32_t periodic[3], int32_t *d_parent,
                               int32_t *d_child, int32_t *d_nbr, int8_t *d_touch, void *stream) {
    if (nblocks <= 0 || nlev <= 0 || nlev > kMaxLevels || !d_level || !d_ijk || !ngb || !periodic || !d_parent ||
        !d_child || !d_nbr || !d_touch)
        return SFM_EINVAL;
    for (int d = 0; d < 3; d++)
        if (ngb[d] <= 0 || ((int64_t)ngb[d] << (nlev - 1)) > ((int64_t)1 << kCoordBits)) return SFM_EINVAL;
    int dev = 0, ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return SFM_EDEVICE;
    }
    if (cudaGetDevice(&dev) != cudaSuccess) return SFM_ECUDA;
    for (const void *p : {(const void *)d_level, (const void *)d_ijk, (const void *)d_parent, (const void *)d_child,
                          (const void *)d_nbr, (const void *)d_touch})
        if (!on_device(p, dev)) return SFM_EINVAL;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) return SFM_EINVAL;
    if (cap != cudaStreamCaptureStatusNone) return SFM_EINVAL;   // the call waits for the stream
    uint64_t slots = 1;
    while (slots < 2 * (uint64_t)nblocks) slots <<= 1;
    LinkTable t{nullptr, nullptr, slots - 1};
    int *err = nullptr;
    if (cudaMallocAsync(&t.keys, slots * sizeof(uint64_t), s) != cudaSuccess ||
        cudaMallocAsync(&t.vals, slots * sizeof(int32_t), s) != cudaSuccess ||
        cudaMallocAsync(&err, sizeof(int), s) != cudaSuccess) {
        cudaGetLastError();
        if (t.keys) cudaFreeAsync(t.keys, s);
        if (t.vals) cudaFreeAsync(t.vals, s);
        return SFM_ENOMEM;
    }
    int herr = 0;
    cudaMemsetAsync(err, 0, sizeof(int), s);
    const unsigned grid = 148 * 4;
    k_link_clear<<<grid, 256, 0, s>>>(t);
    k_link_insert<<<grid, 256, 0, s>>>(t, nblocks, nlev, d_level, d_ijk, make_int3(ngb[0], ngb[1], ngb[2]), err);
    k_link_lookup<<<grid, 256, 0, s>>>(t, nblocks, nlev, d_level, d_ijk, make_int3(ngb[0], ngb[1], ngb[2]),
                                       make_int3(periodic[0] != 0, periodic[1] != 0, periodic[2] != 0), d_parent,
                                       d_child, d_nbr, d_touch, err);
    const cudaError_t launched = cudaGetLastError();
    cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(t.keys, s);
    cudaFreeAsync(t.vals, s);
    cudaFreeAsync(err, s);
    if (launched != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) return SFM_ECUDA;
    return herr ? SFM_EHIER : SFM_OK;
}
