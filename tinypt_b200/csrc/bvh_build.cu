// GPU build of a mesh BVH with the reference's rules (src/bvh.rs:51-242):
// binned SAH over 8 bins on the largest centroid axis when a node has at
// least 16 triangles and a centroid extent above 1e-12, a stable
// reordering of the node's range by bin, otherwise the middle split without
// reordering, leaves of at most 4 triangles, nodes numbered in preorder.
//
// The split decisions are the same arithmetic as the host builder
// (build_mesh_bvh): boxes merge with fmin/fmax, which are exact whatever the
// order of the reduction, and the per-node SAH sweep runs sequentially in
// f64; this translation unit is compiled with -fmad=false so no product is
// fused.  The tree is therefore identical to the host builder's, which the
// tests check node for node.  A child of a SAH split takes its box and
// centroid box as the merge of its side's bin boxes -- the same min/max over
// the same triangles -- so only the root and the children of middle splits
// reduce over their triangles.
//
// Schedule:
//  * nodes above kSmall triangles ("big" nodes) are split level by level:
//    per 4096-triangle chunk the device reduces the bins' counts, boxes and
//    centroid boxes; the host merges the chunks, runs the SAH sweep and hands
//    each chunk its bins' destinations for a stable, ballot-ranked scatter;
//  * nodes of at most kSmall triangles are built whole by one warp each,
//    depth first (binning by ballots, stable partition through a scratch
//    copy, per-bin boxes over the bins' contiguous ranges);
//  * numbering: each warp numbers its subtree in preorder from subtree sizes,
//    the host numbers the big nodes and places the subtrees, and one more
//    kernel writes every node at its preorder index.
#include "bvh_build.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <vector>

namespace tpt {
namespace bvhgpu {

constexpr int kBins = 8;          // SAH_BINS (src/constants.rs:22)
constexpr int kLeaf = 4;          // LEAF_SIZE (src/constants.rs:24)
constexpr int kChunk = 4096;      // triangles per block in the big-node kernels
constexpr int kBlock = 256;       // threads of a big-node block
constexpr int kSmall = 1024;      // nodes this small are built by one warp
constexpr int kSmallStack = 16;   // pending ranges of a warp (<= log2(kSmall) + 1 + 2)
constexpr int kWarps = 4;         // warps (small nodes) per block of the small-node kernels
constexpr unsigned kFull = 0xffffffffu;

struct DBox {
    double lo[3], hi[3];
};

__host__ __device__ inline DBox box_none() {
    const double inf = __builtin_huge_val();
    return DBox{{inf, inf, inf}, {-inf, -inf, -inf}};
}
__host__ __device__ inline void merge(DBox& a, const DBox& b) {
    for (int k = 0; k < 3; ++k) {
        a.lo[k] = fmin(a.lo[k], b.lo[k]);
        a.hi[k] = fmax(a.hi[k], b.hi[k]);
    }
}
__host__ __device__ inline void grow(DBox& a, const double* p) {
    for (int k = 0; k < 3; ++k) {
        a.lo[k] = fmin(a.lo[k], p[k]);
        a.hi[k] = fmax(a.hi[k], p[k]);
    }
}
__host__ __device__ inline double half_area(const DBox& b) {
    const double ex = b.hi[0] - b.lo[0], ey = b.hi[1] - b.lo[1], ez = b.hi[2] - b.lo[2];
    return ex * ey + ey * ez + ez * ex;
}
__host__ __device__ inline int largest_axis(const DBox& cb) {
    const double ex = cb.hi[0] - cb.lo[0], ey = cb.hi[1] - cb.lo[1], ez = cb.hi[2] - cb.lo[2];
    return (ex >= ey && ex >= ez) ? 0 : (ey >= ez ? 1 : 2);
}
// Rust `f as usize` of the bin computation: saturating, NaN -> 0.
__host__ __device__ inline int bin_index(double cv, double minc, double inv_extent) {
    const double f = (cv - minc) * inv_extent * (double)kBins;
    unsigned long long b = (f > 0.0) ? (f >= 1.8446744073709552e19 ? ~0ull : (unsigned long long)f) : 0ull;
    return b >= (unsigned long long)kBins ? kBins - 1 : (int)b;
}

// SAH sweep over the bins (src/bvh.rs:137-176) given each bin's count and
// box: the split bin (0 when no split has finite cost) and, for a split, the
// left count.  Prefix and suffix boxes merge only non-empty bins.
struct Sah {
    int split;      // first bin of the right side; 0 = no finite split
    int left_total;
};
__host__ __device__ inline Sah sah_sweep(const int* cnt, const DBox* bb) {
    double la[kBins], ra[kBins];
    int lc[kBins], rc[kBins];
    DBox acc = box_none();
    int acc_n = 0;
    for (int i = 0; i < kBins; ++i) {
        if (cnt[i] > 0) { merge(acc, bb[i]); acc_n += cnt[i]; }
        la[i] = 2.0 * half_area(acc);
        lc[i] = acc_n;
    }
    acc = box_none();
    acc_n = 0;
    for (int i = kBins - 1; i >= 0; --i) {
        if (cnt[i] > 0) { merge(acc, bb[i]); acc_n += cnt[i]; }
        ra[i] = 2.0 * half_area(acc);
        rc[i] = acc_n;
    }
    double best = __builtin_huge_val();
    int split = 0;
    for (int i = 0; i + 1 < kBins; ++i) {
        if (lc[i] == 0 || rc[i + 1] == 0) continue;
        const double cost = la[i] * (double)lc[i] + ra[i + 1] * (double)rc[i + 1];
        if (cost < best) { best = cost; split = i + 1; }
    }
    if (!isfinite(best)) return Sah{0, 0};
    return Sah{split, lc[split - 1]};
}

__device__ inline DBox load_box(const double* tb, int t) {
    DBox b;
    for (int k = 0; k < 3; ++k) { b.lo[k] = tb[6 * (size_t)t + k]; b.hi[k] = tb[6 * (size_t)t + 3 + k]; }
    return b;
}
// Min / max over the warp; every lane ends with lane 0's result.
__device__ inline void warp_reduce(DBox& b) {
    for (int o = 16; o > 0; o >>= 1)
        for (int k = 0; k < 3; ++k) {
            b.lo[k] = fmin(b.lo[k], __shfl_xor_sync(kFull, b.lo[k], o));
            b.hi[k] = fmax(b.hi[k], __shfl_xor_sync(kFull, b.hi[k], o));
        }
    for (int k = 0; k < 3; ++k) {
        b.lo[k] = __shfl_sync(kFull, b.lo[k], 0);
        b.hi[k] = __shfl_sync(kFull, b.hi[k], 0);
    }
}
// Min / max over a kBlock-thread block; thread 0 holds the result.
__device__ inline void block_reduce(DBox& b, DBox& c, DBox (*sh)[2]) {
    warp_reduce(b);
    warp_reduce(c);
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { sh[w][0] = b; sh[w][1] = c; }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int i = 1; i < kBlock / 32; ++i) { merge(b, sh[i][0]); merge(c, sh[i][1]); }
    __syncthreads();
}
__host__ __device__ inline void store_box(double* o, const DBox& b) {
    for (int k = 0; k < 3; ++k) { o[k] = b.lo[k]; o[3 + k] = b.hi[k]; }
}

// Triangle boxes padded by 1e-9 (Aabb::from_points, src/geometry.rs:70-80)
// and their centres; ord = 0, 1, 2, ...
__global__ void k_tri_boxes(const double* __restrict__ pos, const int32_t* __restrict__ idx, int nt, double* tb,
                            double* cen, int* ord) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nt) return;
    DBox b = box_none();
    for (int k = 0; k < 3; ++k) grow(b, pos + 3 * (size_t)idx[3 * (size_t)i + k]);
    for (int k = 0; k < 3; ++k) {
        b.lo[k] = b.lo[k] - 1e-9;
        b.hi[k] = b.hi[k] + 1e-9;
    }
    for (int k = 0; k < 3; ++k) {
        tb[6 * (size_t)i + k] = b.lo[k];
        tb[6 * (size_t)i + 3 + k] = b.hi[k];
        cen[3 * (size_t)i + k] = (b.lo[k] + b.hi[k]) * 0.5;
    }
    ord[i] = i;
}

// ---- big nodes ----------------------------------------------------------------
struct Chunk { int job, begin, end, pad; };
struct JobBin { int axis, active; double minc, inv_extent; };

// Per chunk: box of the triangle boxes and box of the centres (12 doubles).
__global__ void __launch_bounds__(kBlock) k_chunk_bounds(const Chunk* __restrict__ chunks, const int* __restrict__ ord,
                                                         const double* __restrict__ tb, const double* __restrict__ cen,
                                                         double* out) {
    __shared__ DBox sh[kBlock / 32][2];
    const Chunk c = chunks[blockIdx.x];
    DBox b = box_none(), cb = box_none();
    for (int k = c.begin + (int)threadIdx.x; k < c.end; k += kBlock) {
        const int t = ord[k];
        merge(b, load_box(tb, t));
        grow(cb, cen + 3 * (size_t)t);
    }
    block_reduce(b, cb, sh);
    if (threadIdx.x == 0) {
        store_box(out + 12 * (size_t)blockIdx.x, b);
        store_box(out + 12 * (size_t)blockIdx.x + 6, cb);
    }
}

// Per chunk of a binned node: each triangle's bin (by position in ord), the
// bins' counts, boxes and centroid boxes.
__global__ void __launch_bounds__(kBlock) k_chunk_bins(const Chunk* __restrict__ chunks, const JobBin* __restrict__ jb,
                                                       const int* __restrict__ ord, const double* __restrict__ tb,
                                                       const double* __restrict__ cen, uint8_t* bin_of,
                                                       double* out_box, int* out_cnt) {
    __shared__ DBox sh[kBlock / 32][2];
    __shared__ uint8_t sbin[kChunk];
    __shared__ int cnt[kBins];
    const Chunk c = chunks[blockIdx.x];
    const JobBin j = jb[c.job];
    if (!j.active) return;  // uniform over the block
    if (threadIdx.x < kBins) cnt[threadIdx.x] = 0;
    __syncthreads();
    for (int k = c.begin + (int)threadIdx.x; k < c.end; k += kBlock) {
        const int b = bin_index(cen[3 * (size_t)ord[k] + j.axis], j.minc, j.inv_extent);
        sbin[k - c.begin] = (uint8_t)b;
        bin_of[k] = (uint8_t)b;
        atomicAdd(&cnt[b], 1);
    }
    __syncthreads();
    for (int b = 0; b < kBins; ++b) {
        DBox bb = box_none(), cb = box_none();
        for (int k = c.begin + (int)threadIdx.x; k < c.end; k += kBlock)
            if (sbin[k - c.begin] == b) {
                const int t = ord[k];
                merge(bb, load_box(tb, t));
                grow(cb, cen + 3 * (size_t)t);
            }
        block_reduce(bb, cb, sh);
        if (threadIdx.x == 0) {
            const size_t o = (size_t)blockIdx.x * kBins + b;
            store_box(out_box + 12 * o, bb);
            store_box(out_box + 12 * o + 6, cb);
            out_cnt[o] = cnt[b];
        }
    }
}

// Stable scatter of a partitioned chunk: the chunk's triangles of bin b go
// to dest[b], dest[b] + 1, ... in their order.  1024 threads per block.
__global__ void __launch_bounds__(1024) k_chunk_scatter(const Chunk* __restrict__ chunks, const int* __restrict__ dest,
                                                        const uint8_t* __restrict__ bin_of, const int* __restrict__ ord,
                                                        int* ord2) {
    __shared__ int warp_cnt[32][kBins];
    __shared__ int base[kBins];
    const Chunk c = chunks[blockIdx.x];
    if (dest[(size_t)blockIdx.x * kBins] < 0) return;  // chunk of a node that is not reordered
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x < kBins) base[threadIdx.x] = dest[(size_t)blockIdx.x * kBins + threadIdx.x];
    __syncthreads();
    for (int t0 = c.begin; t0 < c.end; t0 += 1024) {
        const int k = t0 + (int)threadIdx.x;
        const int b = k < c.end ? (int)bin_of[k] : kBins;
        unsigned my_mask = 0;
        for (int q = 0; q < kBins; ++q) {
            const unsigned m = __ballot_sync(kFull, b == q);
            if (lane == 0) warp_cnt[warp][q] = __popc(m);
            if (b == q) my_mask = m;
        }
        __syncthreads();
        if (k < c.end) {
            int before = 0;
            for (int w = 0; w < warp; ++w) before += warp_cnt[w][b];
            const int pos = base[b] + before + __popc(my_mask & ((1u << lane) - 1u));
            ord2[pos] = ord[k];
        }
        __syncthreads();
        if (threadIdx.x < kBins) {
            int tot = 0;
            for (int w = 0; w < 32; ++w) tot += warp_cnt[w][threadIdx.x];
            base[threadIdx.x] += tot;
        }
        __syncthreads();
    }
}

__global__ void k_copy_back(const Chunk* __restrict__ chunks, const int* __restrict__ dest, const int* ord2, int* ord) {
    const Chunk c = chunks[blockIdx.x];
    if (dest[(size_t)blockIdx.x * kBins] < 0) return;
    for (int k = c.begin + (int)threadIdx.x; k < c.end; k += blockDim.x) ord[k] = ord2[k];
}

// ---- small nodes ----------------------------------------------------------------
// A node of at most kSmall triangles with, when its parent was a SAH split,
// its box and centroid box.
struct SmallJob {
    int start, end, has_box, pad;
    DBox bb, cb;
};
struct Pending {
    int s, e, parent, side, depth, has_box;
    DBox bb, cb;
};
// Per-slot arrays of the small-node subtrees.  A subtree over triangles
// [start, end) owns slots 2*start .. 2*start + 2n - 2 (both children of a
// split are non-empty, so it has at most 2n - 1 nodes), filled in creation
// order, parents before children.
struct Slots {
    double* box;   // 6 per slot
    int* lr;       // 2 per slot: child slots, -1 for leaves
    int* sc;       // 2 per slot: leaf start, count
    int* depth;    // per slot: depth below the subtree root
    int* size;     // per slot: nodes in the slot's subtree
    int* pre;      // per slot: preorder index within the subtree
};

// One warp per small node: builds its subtree depth first, descending into
// the smaller child and keeping the larger pending (at most log2(n) + 1
// pending ranges), then numbers the subtree in preorder.
__global__ void __launch_bounds__(32 * kWarps) k_small(const SmallJob* __restrict__ jobs, int n_jobs, int* ord,
                                                       int* scratch, const double* __restrict__ tb,
                                                       const double* __restrict__ cen, Slots sl, int* job_nodes,
                                                       int* flags) {
    __shared__ Pending stk[kWarps][kSmallStack];
    __shared__ uint8_t sbin[kWarps][kSmall];
    __shared__ DBox sbb[kWarps][kBins], scb[kWarps][kBins];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ji = blockIdx.x * kWarps + warp;
    if (ji >= n_jobs) return;  // uniform over the warp
    const SmallJob J = jobs[ji];
    Pending* st = stk[warp];
    uint8_t* bins = sbin[warp];
    const unsigned lt = (1u << lane) - 1u;
    if (lane == 0) st[0] = Pending{J.start, J.end, -1, 0, 0, J.has_box, J.bb, J.cb};
    __syncwarp();
    int sp = 1;
    const int first = 2 * J.start;
    int next = first;
    while (sp > 0) {
        --sp;
        const Pending P = st[sp];
        __syncwarp();
        const int s = P.s, e = P.e, n = e - s;
        DBox bbox = P.bb, cbox = P.cb;
        if (!P.has_box) {
            bbox = box_none();
            cbox = box_none();
            for (int k = s + lane; k < e; k += 32) {
                const int t = ord[k];
                merge(bbox, load_box(tb, t));
                grow(cbox, cen + 3 * (size_t)t);
            }
            warp_reduce(bbox);
            warp_reduce(cbox);
        }
        const int node = next++;
        if (lane == 0) {
            store_box(sl.box + 6 * (size_t)node, bbox);
            sl.lr[2 * (size_t)node] = -1;
            sl.lr[2 * (size_t)node + 1] = -1;
            sl.sc[2 * (size_t)node] = n <= kLeaf ? s : 0;
            sl.sc[2 * (size_t)node + 1] = n <= kLeaf ? n : 0;
            sl.depth[node] = P.depth;
            if (P.parent >= 0) sl.lr[2 * (size_t)P.parent + P.side] = node;
        }
        if (n <= kLeaf) continue;
        const int axis = largest_axis(cbox);
        int mid = s + n / 2;
        bool boxed = false;
        DBox lb = box_none(), lcb = box_none(), rb = box_none(), rcb = box_none();
        const double minc = cbox.lo[axis], extent = cbox.hi[axis] - minc;
        if (n >= kBins * 2 && extent > 1e-12) {
            const double inv_extent = 1.0 / extent;
            int cnt[kBins];
            for (int q = 0; q < kBins; ++q) cnt[q] = 0;
            for (int k0 = s; k0 < e; k0 += 32) {
                const int k = k0 + lane;
                int b = kBins;
                if (k < e) {
                    b = bin_index(cen[3 * (size_t)ord[k] + axis], minc, inv_extent);
                    bins[k - s] = (uint8_t)b;
                }
                for (int q = 0; q < kBins; ++q) cnt[q] += __popc(__ballot_sync(kFull, b == q));
            }
            __syncwarp();
            // stable partition by bin into scratch[s, e)
            int run[kBins];
            for (int q = 0, acc = s; q < kBins; ++q) { run[q] = acc; acc += cnt[q]; }
            for (int k0 = s; k0 < e; k0 += 32) {
                const int k = k0 + lane;
                const int b = k < e ? (int)bins[k - s] : kBins;
                int pos = 0;
                for (int q = 0; q < kBins; ++q) {
                    const unsigned m = __ballot_sync(kFull, b == q);
                    if (b == q) pos = run[q] + __popc(m & lt);
                    run[q] += __popc(m);
                }
                if (k < e) scratch[pos] = ord[k];
            }
            __syncwarp();
            // bin boxes over the bins' contiguous ranges of scratch
            for (int q = 0, off = s; q < kBins; off += cnt[q], ++q) {
                DBox qb = box_none(), qc = box_none();
                if (cnt[q] > 0) {
                    for (int k = off + lane; k < off + cnt[q]; k += 32) {
                        const int t = scratch[k];
                        merge(qb, load_box(tb, t));
                        grow(qc, cen + 3 * (size_t)t);
                    }
                    warp_reduce(qb);
                    warp_reduce(qc);
                }
                if (lane == 0) { sbb[warp][q] = qb; scb[warp][q] = qc; }
            }
            __syncwarp();
            const Sah sah = sah_sweep(cnt, sbb[warp]);
            if (sah.split > 0) {
                for (int k = s + lane; k < e; k += 32) ord[k] = scratch[k];
                __syncwarp();
                if (sah.left_total > 0 && sah.left_total < n) {
                    mid = s + sah.left_total;
                    for (int q = 0; q < kBins; ++q) {
                        if (q < sah.split) { merge(lb, sbb[warp][q]); merge(lcb, scb[warp][q]); }
                        else { merge(rb, sbb[warp][q]); merge(rcb, scb[warp][q]); }
                    }
                    boxed = true;
                }
            }
        }
        if (sp + 2 > kSmallStack) {  // cannot happen while kSmall <= 2^12; kept as a guard
            if (lane == 0) atomicOr(flags, 1);
            return;
        }
        const bool left_small = (mid - s) <= (e - mid);
        if (lane == 0) {
            const Pending L{s, mid, node, 0, P.depth + 1, boxed ? 1 : 0, lb, lcb};
            const Pending R{mid, e, node, 1, P.depth + 1, boxed ? 1 : 0, rb, rcb};
            st[sp] = left_small ? R : L;
            st[sp + 1] = left_small ? L : R;
        }
        __syncwarp();
        sp += 2;
    }
    // subtree sizes (children come after parents) and preorder indices
    if (lane == 0) {
        for (int slot = next - 1; slot >= first; --slot) {
            const int l = sl.lr[2 * (size_t)slot], r = sl.lr[2 * (size_t)slot + 1];
            sl.size[slot] = l < 0 ? 1 : 1 + sl.size[l] + sl.size[r];
        }
        sl.pre[first] = 0;
        for (int slot = first; slot < next; ++slot) {
            const int l = sl.lr[2 * (size_t)slot], r = sl.lr[2 * (size_t)slot + 1];
            if (l < 0) continue;
            sl.pre[l] = sl.pre[slot] + 1;
            sl.pre[r] = sl.pre[slot] + 1 + sl.size[l];
        }
        job_nodes[ji] = next - first;
    }
}

// Writes each small subtree's nodes at base + local preorder index, and the
// leaf order as int64.  One warp per small node.
__global__ void __launch_bounds__(32 * kWarps) k_emit(const SmallJob* __restrict__ jobs, int n_jobs,
                                                      const int* __restrict__ job_base, const int* __restrict__ job_depth,
                                                      const int* __restrict__ job_nodes, Slots sl,
                                                      const int* __restrict__ ord, double* out_box, int32_t* out_lr,
                                                      uint32_t* out_sc, int64_t* out_idx, int* max_depth) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ji = blockIdx.x * kWarps + warp;
    if (ji >= n_jobs) return;
    const SmallJob J = jobs[ji];
    const int base = job_base[ji], d0 = job_depth[ji], first = 2 * J.start, count = job_nodes[ji];
    int md = 0;
    for (int slot = first + lane; slot < first + count; slot += 32) {
        const size_t p = (size_t)base + (size_t)sl.pre[slot];
        for (int k = 0; k < 6; ++k) out_box[6 * p + k] = sl.box[6 * (size_t)slot + k];
        const int l = sl.lr[2 * (size_t)slot], r = sl.lr[2 * (size_t)slot + 1];
        out_lr[2 * p] = l < 0 ? -1 : base + sl.pre[l];
        out_lr[2 * p + 1] = r < 0 ? -1 : base + sl.pre[r];
        out_sc[2 * p] = (uint32_t)sl.sc[2 * (size_t)slot];
        out_sc[2 * p + 1] = (uint32_t)sl.sc[2 * (size_t)slot + 1];
        md = max(md, d0 + sl.depth[slot]);
    }
    for (int o = 16; o > 0; o >>= 1) md = max(md, __shfl_xor_sync(kFull, md, o));
    if (lane == 0) atomicMax(max_depth, md);
    for (int k = J.start + lane; k < J.end; k += 32) out_idx[k] = ord[k];
}

// ---- host driver --------------------------------------------------------------
struct CudaFail : std::runtime_error {
    cudaError_t code;
    CudaFail(cudaError_t c, const std::string& w) : std::runtime_error(w), code(c) {}
};
void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaFail(e, std::string(what) + ": " + cudaGetErrorString(e));
}

// Device allocations of one build, freed together.
struct DevMem {
    std::vector<void*> ptrs;
    ~DevMem() { for (void* p : ptrs) cudaFree(p); }
    template <class T>
    T* alloc(size_t n) {
        void* p = nullptr;
        ck(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)), "device allocation");
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
    template <class T>
    T* upload(const std::vector<T>& v) {
        T* d = alloc<T>(v.size());
        if (!v.empty()) ck(cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
        return d;
    }
};

// A child of a big node: another big node (index into the big list) or a
// small node (index into the small list).
struct Child {
    bool small = false;
    int index = -1;
};
struct BigNode {
    DBox box;
    Child left, right;
};

}  // namespace bvhgpu

int build_mesh_bvh_gpu(const double* positions, int64_t n_vertices, const int32_t* tri_idx, int64_t n_tris,
                       const std::function<GpuBvhSink(int64_t n_nodes)>& sink, int* max_depth_out,
                       int64_t* n_nodes_out, std::string* err) {
    using namespace bvhgpu;
    if (n_tris < 0 || n_vertices < 0) throw std::runtime_error("bad mesh");
    for (int64_t i = 0; i < 3 * n_tris; ++i)
        if (tri_idx[i] < 0 || tri_idx[i] >= n_vertices) throw std::runtime_error("triangle vertex index out of range");
    if (n_tris >= (1ll << 30)) throw std::runtime_error("mesh has too many triangles for the device builder");
    const int nt = (int)n_tris;
    if (max_depth_out) *max_depth_out = 0;
    if (n_nodes_out) *n_nodes_out = 0;
    if (nt == 0) {
        sink(0);
        return kGpuBvhOk;
    }
    try {
        // The fixed-size arrays of the build come from one allocation.
        DevMem mem;
        const size_t T = (size_t)nt;
        const size_t sizes[] = {24 * (size_t)n_vertices, 12 * T, 48 * T, 24 * T, 4 * T, 4 * T, T, 8,
                                96 * T, 16 * T, 16 * T, 8 * T, 8 * T, 8 * T};
        size_t total = 0;
        for (size_t b : sizes) total += (b + 255) & ~(size_t)255;
        char* arena = mem.alloc<char>(total);
        size_t off = 0, next_size = 0;
        auto take = [&]() {
            char* r = arena + off;
            off += (sizes[next_size++] + 255) & ~(size_t)255;
            return (void*)r;
        };
        double* d_pos = (double*)take();
        int32_t* d_idx = (int32_t*)take();
        double* d_tb = (double*)take();
        double* d_cen = (double*)take();
        int* d_ord = (int*)take();
        int* d_ord2 = (int*)take();
        uint8_t* d_bin = (uint8_t*)take();
        int* d_flags = (int*)take();  // [0] stack guard, [1] max depth
        ck(cudaMemcpy(d_pos, positions, 3 * (size_t)n_vertices * sizeof(double), cudaMemcpyHostToDevice), "upload");
        ck(cudaMemcpy(d_idx, tri_idx, 3 * (size_t)nt * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
        ck(cudaMemset(d_flags, 0, 2 * sizeof(int)), "memset");
        k_tri_boxes<<<(nt + 255) / 256, 256>>>(d_pos, d_idx, nt, d_tb, d_cen, d_ord);
        ck(cudaGetLastError(), "triangle boxes");

        std::vector<BigNode> big;
        std::vector<SmallJob> small;
        struct BigJob {
            int start, end, node, has_box;
            DBox bb, cb;
        };
        std::vector<BigJob> level, cur;
        auto make_child = [&](int s, int e, bool has_box, const DBox& bb, const DBox& cb) -> Child {
            if (e - s > kSmall) {
                big.emplace_back();
                level.push_back(BigJob{s, e, (int)big.size() - 1, has_box ? 1 : 0, bb, cb});
                return Child{false, (int)big.size() - 1};
            }
            small.push_back(SmallJob{s, e, has_box ? 1 : 0, 0, bb, cb});
            return Child{true, (int)small.size() - 1};
        };
        const Child root = make_child(0, nt, false, box_none(), box_none());

        // Big nodes, one level per pass.  Every level strictly shrinks each
        // big node, so the loop ends; a lopsided tree (SAH peeling a few
        // triangles per split) takes many levels of a few launches each.
        DevMem lvl;
        Chunk* d_chunks = nullptr;
        size_t chunk_cap = 0, job_cap = 0;
        double *d_part = nullptr, *d_bbox = nullptr;
        int *d_bcnt = nullptr, *d_dest = nullptr;
        JobBin* d_jb = nullptr;
        while (!level.empty()) {
            cur.swap(level);
            level.clear();
            std::vector<Chunk> chunks;
            bool need_bounds = false;
            for (size_t j = 0; j < cur.size(); ++j) {
                need_bounds |= !cur[j].has_box;
                for (int b = cur[j].start; b < cur[j].end; b += kChunk)
                    chunks.push_back(Chunk{(int)j, b, std::min(b + kChunk, cur[j].end), 0});
            }
            const size_t nc = chunks.size();
            if (nc > chunk_cap) {
                chunk_cap = 2 * nc;
                d_chunks = lvl.alloc<Chunk>(chunk_cap);
                d_part = lvl.alloc<double>(12 * chunk_cap);
                d_bbox = lvl.alloc<double>(12 * kBins * chunk_cap);
                d_bcnt = lvl.alloc<int>(kBins * chunk_cap);
                d_dest = lvl.alloc<int>(kBins * chunk_cap);
            }
            if (cur.size() > job_cap) {
                job_cap = 2 * cur.size();
                d_jb = lvl.alloc<JobBin>(job_cap);
            }
            ck(cudaMemcpy(d_chunks, chunks.data(), nc * sizeof(Chunk), cudaMemcpyHostToDevice), "chunks");
            if (need_bounds) {
                k_chunk_bounds<<<(unsigned)nc, kBlock>>>(d_chunks, d_ord, d_tb, d_cen, d_part);
                ck(cudaGetLastError(), "chunk bounds");
                std::vector<double> part(12 * nc);
                ck(cudaMemcpy(part.data(), d_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost), "bounds");
                for (BigJob& J : cur)
                    if (!J.has_box) J.bb = J.cb = box_none();
                for (size_t c = 0; c < nc; ++c) {
                    BigJob& J = cur[(size_t)chunks[c].job];
                    if (J.has_box) continue;
                    const double* p = &part[12 * c];
                    merge(J.bb, DBox{{p[0], p[1], p[2]}, {p[3], p[4], p[5]}});
                    merge(J.cb, DBox{{p[6], p[7], p[8]}, {p[9], p[10], p[11]}});
                }
            }
            std::vector<JobBin> jb(cur.size());
            for (size_t j = 0; j < cur.size(); ++j) {
                big[(size_t)cur[j].node].box = cur[j].bb;
                const DBox& cb = cur[j].cb;
                const int axis = largest_axis(cb);
                const double minc = cb.lo[axis], extent = cb.hi[axis] - minc;
                jb[j] = JobBin{axis, extent > 1e-12 ? 1 : 0, minc, extent > 1e-12 ? 1.0 / extent : 0.0};
            }
            ck(cudaMemcpy(d_jb, jb.data(), jb.size() * sizeof(JobBin), cudaMemcpyHostToDevice), "job bins");
            k_chunk_bins<<<(unsigned)nc, kBlock>>>(d_chunks, d_jb, d_ord, d_tb, d_cen, d_bin, d_bbox, d_bcnt);
            ck(cudaGetLastError(), "chunk bins");
            std::vector<double> cbins(12 * kBins * nc);
            std::vector<int> ccnt(kBins * nc);
            ck(cudaMemcpy(cbins.data(), d_bbox, cbins.size() * sizeof(double), cudaMemcpyDeviceToHost), "bins");
            ck(cudaMemcpy(ccnt.data(), d_bcnt, ccnt.size() * sizeof(int), cudaMemcpyDeviceToHost), "bins");
            // per node: merge the chunks' bins, SAH sweep, split; per chunk:
            // where each bin's triangles go
            std::vector<int> dest(kBins * nc, -1);
            struct Split { int mid; bool boxed; DBox lb, lcb, rb, rcb; };
            std::vector<Split> splits(cur.size());
            size_t c0 = 0;
            for (size_t j = 0; j < cur.size(); ++j) {
                const int s = cur[j].start, e = cur[j].end, n = e - s;
                size_t c1 = c0;
                while (c1 < nc && chunks[c1].job == (int)j) ++c1;
                Split& S = splits[j];
                S = Split{s + n / 2, false, box_none(), box_none(), box_none(), box_none()};
                if (jb[j].active) {  // n > kSmall >= 16
                    DBox bb[kBins], cb[kBins];
                    int cnt[kBins];
                    for (int b = 0; b < kBins; ++b) { bb[b] = box_none(); cb[b] = box_none(); cnt[b] = 0; }
                    for (size_t c = c0; c < c1; ++c)
                        for (int b = 0; b < kBins; ++b) {
                            const double* p = &cbins[12 * (c * kBins + b)];
                            merge(bb[b], DBox{{p[0], p[1], p[2]}, {p[3], p[4], p[5]}});
                            merge(cb[b], DBox{{p[6], p[7], p[8]}, {p[9], p[10], p[11]}});
                            cnt[b] += ccnt[c * kBins + b];
                        }
                    const Sah sah = sah_sweep(cnt, bb);
                    if (sah.split > 0) {
                        int run[kBins];
                        for (int b = 0, acc = s; b < kBins; ++b) { run[b] = acc; acc += cnt[b]; }
                        for (size_t c = c0; c < c1; ++c)
                            for (int b = 0; b < kBins; ++b) {
                                dest[c * kBins + b] = run[b];
                                run[b] += ccnt[c * kBins + b];
                            }
                        if (sah.left_total > 0 && sah.left_total < n) {
                            S.mid = s + sah.left_total;
                            S.boxed = true;
                            for (int b = 0; b < kBins; ++b) {
                                if (b < sah.split) { merge(S.lb, bb[b]); merge(S.lcb, cb[b]); }
                                else { merge(S.rb, bb[b]); merge(S.rcb, cb[b]); }
                            }
                        }
                    }
                }
                c0 = c1;
            }
            ck(cudaMemcpy(d_dest, dest.data(), dest.size() * sizeof(int), cudaMemcpyHostToDevice), "dest");
            k_chunk_scatter<<<(unsigned)nc, 1024>>>(d_chunks, d_dest, d_bin, d_ord, d_ord2);
            ck(cudaGetLastError(), "scatter");
            k_copy_back<<<(unsigned)nc, 256>>>(d_chunks, d_dest, d_ord2, d_ord);
            ck(cudaGetLastError(), "copy back");
            for (size_t j = 0; j < cur.size(); ++j) {
                const Split& S = splits[j];
                const Child l = make_child(cur[j].start, S.mid, S.boxed, S.lb, S.lcb);
                const Child r = make_child(S.mid, cur[j].end, S.boxed, S.rb, S.rcb);
                big[(size_t)cur[j].node].left = l;
                big[(size_t)cur[j].node].right = r;
            }
        }

        // Small nodes: one warp each.
        const int n_small = (int)small.size();
        Slots sl;
        sl.box = (double*)take();
        sl.lr = (int*)take();
        sl.sc = (int*)take();
        sl.depth = (int*)take();
        sl.size = (int*)take();
        sl.pre = (int*)take();
        SmallJob* d_small = mem.upload(small);
        int* d_job_nodes = mem.alloc<int>((size_t)n_small);
        const unsigned small_blocks = (unsigned)((n_small + kWarps - 1) / kWarps);
        k_small<<<small_blocks, 32 * kWarps>>>(d_small, n_small, d_ord, d_ord2, d_tb, d_cen, sl, d_job_nodes, d_flags);
        ck(cudaGetLastError(), "small nodes");
        std::vector<int> job_nodes((size_t)n_small);
        ck(cudaMemcpy(job_nodes.data(), d_job_nodes, job_nodes.size() * sizeof(int), cudaMemcpyDeviceToHost),
           "node counts");
        int guard = 0;
        ck(cudaMemcpy(&guard, d_flags, sizeof(int), cudaMemcpyDeviceToHost), "flags");
        if (guard) {
            if (err) *err = "a small node overflowed its pending-range stack";
            return kGpuBvhUseHost;
        }

        // Preorder over the big nodes: sizes bottom up (big nodes were made
        // parents first), then indices and depths top down.
        const size_t nb = big.size();
        std::vector<int64_t> bsize(nb), bpre(nb);
        std::vector<int> bdepth(nb);
        auto child_size = [&](const Child& c) -> int64_t {
            return c.small ? (int64_t)job_nodes[(size_t)c.index] : bsize[(size_t)c.index];
        };
        for (size_t i = nb; i-- > 0;) bsize[i] = 1 + child_size(big[i].left) + child_size(big[i].right);
        const int64_t n_nodes = root.small ? (int64_t)job_nodes[0] : bsize[0];
        std::vector<int> job_base((size_t)n_small), job_depth((size_t)n_small);
        auto place = [&](const Child& c, int64_t pre, int depth) {
            if (c.small) {
                job_base[(size_t)c.index] = (int)pre;
                job_depth[(size_t)c.index] = depth;
            } else {
                bpre[(size_t)c.index] = pre;
                bdepth[(size_t)c.index] = depth;
            }
        };
        place(root, 0, 1);
        int max_depth = 0;
        for (size_t i = 0; i < nb; ++i) {
            place(big[i].left, bpre[i] + 1, bdepth[i] + 1);
            place(big[i].right, bpre[i] + 1 + child_size(big[i].left), bdepth[i] + 1);
            max_depth = std::max(max_depth, bdepth[i]);
        }

        const GpuBvhSink out = sink(n_nodes);
        if (out.bbox || out.left_right || out.start_count || out.indices) {
            const size_t nn = (size_t)n_nodes;
            const size_t o1 = (48 * nn + 255) & ~(size_t)255, o2 = o1 + ((8 * nn + 255) & ~(size_t)255),
                         o3 = o2 + ((8 * nn + 255) & ~(size_t)255);
            char* out_arena = mem.alloc<char>(o3 + 8 * T);
            double* d_obox = (double*)out_arena;
            int32_t* d_olr = (int32_t*)(out_arena + o1);
            uint32_t* d_osc = (uint32_t*)(out_arena + o2);
            int64_t* d_oidx = (int64_t*)(out_arena + o3);
            int* d_base = mem.upload(job_base);
            int* d_depth = mem.upload(job_depth);
            k_emit<<<small_blocks, 32 * kWarps>>>(d_small, n_small, d_base, d_depth, d_job_nodes, sl, d_ord, d_obox,
                                                  d_olr, d_osc, d_oidx, d_flags + 1);
            ck(cudaGetLastError(), "emit");
            if (out.bbox)
                ck(cudaMemcpy(out.bbox, d_obox, 6 * (size_t)n_nodes * sizeof(double), cudaMemcpyDeviceToHost), "nodes");
            if (out.left_right)
                ck(cudaMemcpy(out.left_right, d_olr, 2 * (size_t)n_nodes * sizeof(int32_t), cudaMemcpyDeviceToHost),
                   "nodes");
            if (out.start_count)
                ck(cudaMemcpy(out.start_count, d_osc, 2 * (size_t)n_nodes * sizeof(uint32_t), cudaMemcpyDeviceToHost),
                   "nodes");
            if (out.indices)
                ck(cudaMemcpy(out.indices, d_oidx, (size_t)nt * sizeof(int64_t), cudaMemcpyDeviceToHost), "order");
            int small_depth = 0;
            ck(cudaMemcpy(&small_depth, d_flags + 1, sizeof(int), cudaMemcpyDeviceToHost), "depth");
            max_depth = std::max(max_depth, small_depth);
            // the big nodes, written over their places
            auto pre_of = [&](const Child& c) -> int32_t {
                return (int32_t)(c.small ? job_base[(size_t)c.index] : bpre[(size_t)c.index]);
            };
            for (size_t i = 0; i < nb; ++i) {
                const size_t p = (size_t)bpre[i];
                if (out.bbox) store_box(out.bbox + 6 * p, big[i].box);
                if (out.left_right) {
                    out.left_right[2 * p] = pre_of(big[i].left);
                    out.left_right[2 * p + 1] = pre_of(big[i].right);
                }
                if (out.start_count) {
                    out.start_count[2 * p] = 0;
                    out.start_count[2 * p + 1] = 0;
                }
            }
        }
        if (max_depth_out) *max_depth_out = max_depth;
        if (n_nodes_out) *n_nodes_out = n_nodes;
        return kGpuBvhOk;
    } catch (const CudaFail& e) {
        if (err) *err = e.what();
        cudaGetLastError();
        return e.code == cudaErrorMemoryAllocation ? kGpuBvhNoMemory : kGpuBvhCudaError;
    }
}

int build_mesh_bvh_gpu(const double* positions, int64_t n_vertices, const int32_t* tri_idx, int64_t n_tris,
                       HostBvh& out, std::string* err) {
    out = HostBvh{};
    int depth = 0;
    int64_t n = 0;
    const int rc = build_mesh_bvh_gpu(
        positions, n_vertices, tri_idx, n_tris,
        [&](int64_t n_nodes) {
            out.bbox.resize(6 * (size_t)n_nodes);
            out.left_right.resize(2 * (size_t)n_nodes);
            out.start_count.resize(2 * (size_t)n_nodes);
            out.indices.resize((size_t)n_tris);
            return GpuBvhSink{out.bbox.data(), out.left_right.data(), out.start_count.data(), out.indices.data()};
        },
        &depth, &n, err);
    if (rc == kGpuBvhOk) out.max_depth = depth;
    return rc;
}

}  // namespace tpt
