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
// tests check node for node.
//
// Schedule: nodes with more than kSmall triangles ("big" nodes) are split
// level by level, each level reducing boxes and bin counts over 4096-element
// chunks on the device and taking the per-node decisions on the host; the
// stable partition by bin is a ballot-ranked scatter.  Nodes of at most
// kSmall triangles are built whole by one thread each, depth first.  The
// host finally numbers the nodes in preorder.
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
constexpr int kChunk = 4096;      // elements per block in the big-node kernels
constexpr int kSmall = 1024;      // nodes this small are built by one thread
constexpr int kSmallStack = 32;   // pending siblings of a small-node thread (<= log2(kSmall) + 1)
constexpr int kBlock = 256;

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
// Rust `f as usize` of the bin computation: saturating, NaN -> 0.
__host__ __device__ inline int bin_index(double cv, double minc, double inv_extent) {
    const double f = (cv - minc) * inv_extent * (double)kBins;
    unsigned long long b = (f > 0.0) ? (f >= 1.8446744073709552e19 ? ~0ull : (unsigned long long)f) : 0ull;
    return b >= (unsigned long long)kBins ? kBins - 1 : (int)b;
}
__device__ inline DBox load_box(const double* tb, int t) {
    DBox b;
    for (int k = 0; k < 3; ++k) { b.lo[k] = tb[6 * (size_t)t + k]; b.hi[k] = tb[6 * (size_t)t + 3 + k]; }
    return b;
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

struct Chunk { int job, begin, end, pad; };
struct JobBin { int axis, active; double minc, inv_extent; };

// Block-wide min / max of a box held per thread (shared scratch of 6*kBlock doubles).
__device__ void block_reduce_box(DBox& b, double* sh) {
    for (int k = 0; k < 3; ++k) {
        sh[k * kBlock + threadIdx.x] = b.lo[k];
        sh[(3 + k) * kBlock + threadIdx.x] = b.hi[k];
    }
    __syncthreads();
    for (int s = kBlock / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            for (int k = 0; k < 3; ++k) {
                double* lo = sh + k * kBlock;
                double* hi = sh + (3 + k) * kBlock;
                lo[threadIdx.x] = fmin(lo[threadIdx.x], lo[threadIdx.x + s]);
                hi[threadIdx.x] = fmax(hi[threadIdx.x], hi[threadIdx.x + s]);
            }
        }
        __syncthreads();
    }
    for (int k = 0; k < 3; ++k) { b.lo[k] = sh[k * kBlock]; b.hi[k] = sh[(3 + k) * kBlock]; }
    __syncthreads();
}

// Per chunk: box of the triangle boxes and box of the centres.
__global__ void __launch_bounds__(kBlock) k_chunk_bounds(const Chunk* __restrict__ chunks, const int* __restrict__ ord,
                                                         const double* __restrict__ tb, const double* __restrict__ cen,
                                                         double* out) {
    __shared__ double sh[6 * kBlock];
    const Chunk c = chunks[blockIdx.x];
    DBox b = box_none(), cb = box_none();
    for (int k = c.begin + (int)threadIdx.x; k < c.end; k += kBlock) {
        const int t = ord[k];
        merge(b, load_box(tb, t));
        grow(cb, cen + 3 * (size_t)t);
    }
    block_reduce_box(b, sh);
    block_reduce_box(cb, sh);
    if (threadIdx.x == 0) {
        double* o = out + 12 * (size_t)blockIdx.x;
        for (int k = 0; k < 3; ++k) {
            o[k] = b.lo[k]; o[3 + k] = b.hi[k]; o[6 + k] = cb.lo[k]; o[9 + k] = cb.hi[k];
        }
    }
}

// Per chunk of a binned node: each element's bin (by position), the bins'
// triangle counts and boxes.
__global__ void __launch_bounds__(kBlock) k_chunk_bins(const Chunk* __restrict__ chunks, const JobBin* __restrict__ jb,
                                                       const int* __restrict__ ord, const double* __restrict__ tb,
                                                       const double* __restrict__ cen, uint8_t* bin_of,
                                                       double* out_box, int* out_cnt) {
    __shared__ double sh[6 * kBlock];
    __shared__ int cnt[kBins];
    const Chunk c = chunks[blockIdx.x];
    const JobBin j = jb[c.job];
    if (threadIdx.x < kBins) cnt[threadIdx.x] = 0;
    __syncthreads();
    if (!j.active) return;  // uniform over the block
    for (int k = c.begin + (int)threadIdx.x; k < c.end; k += kBlock) {
        const int t = ord[k];
        const int b = bin_index(cen[3 * (size_t)t + j.axis], j.minc, j.inv_extent);
        bin_of[k] = (uint8_t)b;
        atomicAdd(&cnt[b], 1);
    }
    __syncthreads();
    for (int b = 0; b < kBins; ++b) {
        DBox bb = box_none();
        for (int k = c.begin + (int)threadIdx.x; k < c.end; k += kBlock)
            if (bin_of[k] == b) merge(bb, load_box(tb, ord[k]));
        block_reduce_box(bb, sh);
        if (threadIdx.x == 0) {
            double* o = out_box + 6 * ((size_t)blockIdx.x * kBins + b);
            for (int k = 0; k < 3; ++k) { o[k] = bb.lo[k]; o[3 + k] = bb.hi[k]; }
            out_cnt[(size_t)blockIdx.x * kBins + b] = cnt[b];
        }
    }
}

// Stable scatter of a partitioned chunk: element k of bin b goes to
// dest[b] + (elements of bin b before it in the chunk).  Block of 1024
// threads, one element per thread per tile.
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
            const unsigned m = __ballot_sync(0xffffffffu, b == q);
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

// A node of at most kSmall triangles, built whole by one thread with the
// host builder's steps.  Its nodes take slots 2*start .. 2*start + 2n - 2
// (both children of a split are non-empty, so a subtree over n triangles has
// at most 2n - 1 nodes).  The thread descends into the smaller child first
// and keeps the larger one pending, so at most log2(n) + 1 ranges wait; the
// order in which it visits nodes does not matter, the host numbers them in
// preorder from the child links.
struct SmallJob { int start, end; };
__global__ void k_small(const SmallJob* __restrict__ jobs, int n_jobs, int* ord, int* scratch, uint8_t* bin_of,
                        const double* __restrict__ tb, const double* __restrict__ cen, double* nbox, int* nlr,
                        int* nsc, int* flags) {
    const int ji = blockIdx.x * blockDim.x + threadIdx.x;
    if (ji >= n_jobs) return;
    const SmallJob J = jobs[ji];
    int st_s[kSmallStack], st_e[kSmallStack], st_p[kSmallStack], st_side[kSmallStack];
    int sp = 0;
    st_s[0] = J.start; st_e[0] = J.end; st_p[0] = -1; st_side[0] = 0;
    sp = 1;
    int next = 2 * J.start;
    while (sp > 0) {
        --sp;
        const int s = st_s[sp], e = st_e[sp], parent = st_p[sp], side = st_side[sp];
        const int n = e - s;
        DBox bbox = box_none(), cbox = box_none();
        for (int k = s; k < e; ++k) {
            const int t = ord[k];
            merge(bbox, load_box(tb, t));
            grow(cbox, cen + 3 * (size_t)t);
        }
        const int node = next++;
        for (int k = 0; k < 3; ++k) { nbox[6 * (size_t)node + k] = bbox.lo[k]; nbox[6 * (size_t)node + 3 + k] = bbox.hi[k]; }
        nlr[2 * (size_t)node] = -1; nlr[2 * (size_t)node + 1] = -1;
        nsc[2 * (size_t)node] = 0; nsc[2 * (size_t)node + 1] = 0;
        if (parent >= 0) nlr[2 * (size_t)parent + side] = node;
        if (n <= kLeaf) {
            nsc[2 * (size_t)node] = s;
            nsc[2 * (size_t)node + 1] = n;
            continue;
        }
        const double ext[3] = {cbox.hi[0] - cbox.lo[0], cbox.hi[1] - cbox.lo[1], cbox.hi[2] - cbox.lo[2]};
        const int axis = (ext[0] >= ext[1] && ext[0] >= ext[2]) ? 0 : (ext[1] >= ext[2] ? 1 : 2);
        int mid = s + n / 2;
        if (n >= kBins * 2) {
            const double minc = cbox.lo[axis], maxc = cbox.hi[axis];
            const double extent = maxc - minc;
            if (extent > 1e-12) {
                const double inv_extent = 1.0 / extent;
                DBox bbin[kBins];
                int cnt[kBins];
                for (int b = 0; b < kBins; ++b) { bbin[b] = box_none(); cnt[b] = 0; }
                for (int k = s; k < e; ++k) {
                    const int t = ord[k];
                    const int b = bin_index(cen[3 * (size_t)t + axis], minc, inv_extent);
                    bin_of[k] = (uint8_t)b;
                    merge(bbin[b], load_box(tb, t));
                    cnt[b] += 1;
                }
                DBox lbox[kBins], rbox[kBins];
                int lcnt[kBins], rcnt[kBins];
                DBox acc = box_none();
                int acc_n = 0;
                for (int i = 0; i < kBins; ++i) {
                    if (cnt[i] > 0) { merge(acc, bbin[i]); acc_n += cnt[i]; }
                    lbox[i] = acc; lcnt[i] = acc_n;
                }
                acc = box_none();
                acc_n = 0;
                for (int i = kBins - 1; i >= 0; --i) {
                    if (cnt[i] > 0) { merge(acc, bbin[i]); acc_n += cnt[i]; }
                    rbox[i] = acc; rcnt[i] = acc_n;
                }
                double best = __builtin_huge_val();
                int split = 0;
                for (int i = 0; i + 1 < kBins; ++i) {
                    const int lc = lcnt[i], rc = rcnt[i + 1];
                    if (lc == 0 || rc == 0) continue;
                    const double la = 2.0 * half_area(lbox[i]);
                    const double ra = 2.0 * half_area(rbox[i + 1]);
                    const double cost = la * (double)lc + ra * (double)rc;
                    if (cost < best) { best = cost; split = i + 1; }
                }
                if (isfinite(best)) {
                    int off[kBins];
                    int run = 0;
                    for (int b = 0; b < kBins; ++b) { off[b] = run; run += cnt[b]; }
                    for (int k = s; k < e; ++k) scratch[s + off[bin_of[k]]++] = ord[k];
                    for (int k = s; k < e; ++k) ord[k] = scratch[k];
                    int left_total = 0;
                    for (int b = 0; b < split; ++b) left_total += cnt[b];
                    if (left_total > 0 && left_total < n) mid = s + left_total;
                }
            }
        }
        if (sp + 2 > kSmallStack) {  // cannot happen while kSmall <= 2^20; kept as a guard
            atomicOr(flags, 1);
            return;
        }
        const bool left_small = (mid - s) <= (e - mid);
        st_s[sp] = left_small ? mid : s; st_e[sp] = left_small ? e : mid;
        st_p[sp] = node; st_side[sp] = left_small ? 1 : 0; ++sp;
        st_s[sp] = left_small ? s : mid; st_e[sp] = left_small ? mid : e;
        st_p[sp] = node; st_side[sp] = left_small ? 0 : 1; ++sp;
    }
}

// ---- host driver --------------------------------------------------------------
struct DevBuf {
    std::vector<void*> ptrs;
    ~DevBuf() { for (void* p : ptrs) cudaFree(p); }
    template <class T>
    T* alloc(size_t n) {
        void* p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) throw std::bad_alloc();
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
};

struct CudaFail : std::runtime_error {
    using std::runtime_error::runtime_error;
};
void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaFail(std::string(what) + ": " + cudaGetErrorString(e));
}

constexpr long long kSmallBase = 1ll << 40;  // node ids of small-node slots: kSmallBase + slot

struct BigNode {
    DBox box;
    long long left = -1, right = -1;
    int start = 0, count = 0;
};

}  // namespace bvhgpu

int build_mesh_bvh_gpu(const double* positions, int64_t n_vertices, const int32_t* tri_idx, int64_t n_tris,
                       HostBvh& out, std::string* err) {
    using namespace bvhgpu;
    out = HostBvh{};
    if (n_tris < 0 || n_vertices < 0) throw std::runtime_error("bad mesh");
    for (int64_t i = 0; i < 3 * n_tris; ++i)
        if (tri_idx[i] < 0 || tri_idx[i] >= n_vertices) throw std::runtime_error("triangle vertex index out of range");
    if (n_tris >= (1ll << 30)) throw std::runtime_error("mesh has too many triangles for the GPU builder");
    const int nt = (int)n_tris;
    if (nt == 0) {
        out = build_mesh_bvh(positions, n_vertices, tri_idx, 0);
        return kGpuBvhOk;
    }
    try {
        DevBuf mem;
        double* d_pos = mem.alloc<double>(3 * (size_t)n_vertices);
        int32_t* d_idx = mem.alloc<int32_t>(3 * (size_t)nt);
        double* d_tb = mem.alloc<double>(6 * (size_t)nt);
        double* d_cen = mem.alloc<double>(3 * (size_t)nt);
        int* d_ord = mem.alloc<int>(nt);
        int* d_ord2 = mem.alloc<int>(nt);
        uint8_t* d_bin = mem.alloc<uint8_t>(nt);
        double* d_nbox = mem.alloc<double>(6 * 2 * (size_t)nt);
        int* d_nlr = mem.alloc<int>(2 * 2 * (size_t)nt);
        int* d_nsc = mem.alloc<int>(2 * 2 * (size_t)nt);
        int* d_flags = mem.alloc<int>(1);
        ck(cudaMemcpy(d_pos, positions, 3 * (size_t)n_vertices * sizeof(double), cudaMemcpyHostToDevice), "upload");
        ck(cudaMemcpy(d_idx, tri_idx, 3 * (size_t)nt * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
        ck(cudaMemset(d_flags, 0, sizeof(int)), "memset");
        k_tri_boxes<<<(nt + 255) / 256, 256>>>(d_pos, d_idx, nt, d_tb, d_cen, d_ord);
        ck(cudaGetLastError(), "triangle boxes");

        std::vector<BigNode> big;
        struct BigJob { int start, end; long long id; };
        std::vector<BigJob> level;
        std::vector<SmallJob> small;
        long long root;
        auto child = [&](int s, int e) -> long long {
            if (e - s > kSmall) {
                big.emplace_back();
                level.push_back(BigJob{s, e, (long long)big.size() - 1});
                return (long long)big.size() - 1;
            }
            small.push_back(SmallJob{s, e});
            return kSmallBase + 2ll * s;
        };
        std::vector<BigJob> cur;
        root = child(0, nt);
        Chunk* d_chunks = nullptr;
        size_t d_chunks_cap = 0;
        double* d_part = nullptr;
        JobBin* d_jb = nullptr;
        size_t d_jb_cap = 0;
        double* d_bbox = nullptr;
        int* d_bcnt = nullptr;
        int* d_dest = nullptr;
        DevBuf lvl;
        // Every level strictly shrinks each big node, so the loop ends; a
        // lopsided tree (SAH peeling a few triangles per split) takes many
        // levels, each a few launches and copies.
        while (!level.empty()) {
            cur.swap(level);
            level.clear();
            std::vector<Chunk> chunks;
            for (size_t j = 0; j < cur.size(); ++j)
                for (int b = cur[j].start; b < cur[j].end; b += kChunk)
                    chunks.push_back(Chunk{(int)j, b, std::min(b + kChunk, cur[j].end), 0});
            const size_t nc = chunks.size();
            if (nc > d_chunks_cap) {
                d_chunks = lvl.alloc<Chunk>(nc);
                d_part = lvl.alloc<double>(12 * nc);
                d_bbox = lvl.alloc<double>(6 * kBins * nc);
                d_bcnt = lvl.alloc<int>(kBins * nc);
                d_dest = lvl.alloc<int>(kBins * nc);
                d_chunks_cap = nc;
            }
            if (cur.size() > d_jb_cap) {
                d_jb = lvl.alloc<JobBin>(cur.size());
                d_jb_cap = cur.size();
            }
            ck(cudaMemcpy(d_chunks, chunks.data(), nc * sizeof(Chunk), cudaMemcpyHostToDevice), "chunks");
            k_chunk_bounds<<<(unsigned)nc, kBlock>>>(d_chunks, d_ord, d_tb, d_cen, d_part);
            ck(cudaGetLastError(), "chunk bounds");
            std::vector<double> part(12 * nc);
            ck(cudaMemcpy(part.data(), d_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost), "bounds");
            std::vector<DBox> jbox(cur.size(), box_none()), jcb(cur.size(), box_none());
            for (size_t c = 0; c < nc; ++c) {
                const double* p = &part[12 * c];
                DBox b{{p[0], p[1], p[2]}, {p[3], p[4], p[5]}}, cb{{p[6], p[7], p[8]}, {p[9], p[10], p[11]}};
                merge(jbox[(size_t)chunks[c].job], b);
                merge(jcb[(size_t)chunks[c].job], cb);
            }
            std::vector<JobBin> jb(cur.size());
            for (size_t j = 0; j < cur.size(); ++j) {
                big[(size_t)cur[j].id].box = jbox[j];
                const DBox& cb = jcb[j];
                const double ext[3] = {cb.hi[0] - cb.lo[0], cb.hi[1] - cb.lo[1], cb.hi[2] - cb.lo[2]};
                const int axis = (ext[0] >= ext[1] && ext[0] >= ext[2]) ? 0 : (ext[1] >= ext[2] ? 1 : 2);
                const double minc = cb.lo[axis], maxc = cb.hi[axis];
                const double extent = maxc - minc;
                jb[j] = JobBin{axis, extent > 1e-12 ? 1 : 0, minc, extent > 1e-12 ? 1.0 / extent : 0.0};
            }
            ck(cudaMemcpy(d_jb, jb.data(), jb.size() * sizeof(JobBin), cudaMemcpyHostToDevice), "job bins");
            k_chunk_bins<<<(unsigned)nc, kBlock>>>(d_chunks, d_jb, d_ord, d_tb, d_cen, d_bin, d_bbox, d_bcnt);
            ck(cudaGetLastError(), "chunk bins");
            std::vector<double> cbox(6 * kBins * nc);
            std::vector<int> ccnt(kBins * nc);
            ck(cudaMemcpy(cbox.data(), d_bbox, cbox.size() * sizeof(double), cudaMemcpyDeviceToHost), "bins");
            ck(cudaMemcpy(ccnt.data(), d_bcnt, ccnt.size() * sizeof(int), cudaMemcpyDeviceToHost), "bins");
            // per node: bins, SAH sweep, split; per chunk: where each bin's elements go
            std::vector<int> dest(kBins * nc, -1);
            std::vector<int> mids(cur.size());
            size_t c0 = 0;
            for (size_t j = 0; j < cur.size(); ++j) {
                const int s = cur[j].start, e = cur[j].end, n = e - s;
                size_t c1 = c0;
                while (c1 < nc && chunks[c1].job == (int)j) ++c1;
                int mid = s + n / 2;
                if (jb[j].active) {  // n > kSmall >= 16
                    DBox bbin[kBins];
                    int cnt[kBins];
                    for (int b = 0; b < kBins; ++b) { bbin[b] = box_none(); cnt[b] = 0; }
                    for (size_t c = c0; c < c1; ++c)
                        for (int b = 0; b < kBins; ++b) {
                            const double* p = &cbox[6 * (c * kBins + b)];
                            merge(bbin[b], DBox{{p[0], p[1], p[2]}, {p[3], p[4], p[5]}});
                            cnt[b] += ccnt[c * kBins + b];
                        }
                    DBox lbox[kBins], rbox[kBins];
                    int lcnt[kBins], rcnt[kBins];
                    DBox acc = box_none();
                    int acc_n = 0;
                    for (int i = 0; i < kBins; ++i) {
                        if (cnt[i] > 0) { merge(acc, bbin[i]); acc_n += cnt[i]; }
                        lbox[i] = acc; lcnt[i] = acc_n;
                    }
                    acc = box_none();
                    acc_n = 0;
                    for (int i = kBins - 1; i >= 0; --i) {
                        if (cnt[i] > 0) { merge(acc, bbin[i]); acc_n += cnt[i]; }
                        rbox[i] = acc; rcnt[i] = acc_n;
                    }
                    double best = std::numeric_limits<double>::infinity();
                    int split = 0;
                    for (int i = 0; i + 1 < kBins; ++i) {
                        const int lc = lcnt[i], rc = rcnt[i + 1];
                        if (lc == 0 || rc == 0) continue;
                        const double la = 2.0 * half_area(lbox[i]);
                        const double ra = 2.0 * half_area(rbox[i + 1]);
                        const double cost = la * (double)lc + ra * (double)rc;
                        if (cost < best) { best = cost; split = i + 1; }
                    }
                    if (std::isfinite(best)) {
                        int run[kBins];
                        int acc2 = s;
                        for (int b = 0; b < kBins; ++b) { run[b] = acc2; acc2 += cnt[b]; }
                        for (size_t c = c0; c < c1; ++c)
                            for (int b = 0; b < kBins; ++b) {
                                dest[c * kBins + b] = run[b];
                                run[b] += ccnt[c * kBins + b];
                            }
                        int left_total = 0;
                        for (int b = 0; b < split; ++b) left_total += cnt[b];
                        if (left_total > 0 && left_total < n) mid = s + left_total;
                    }
                }
                mids[j] = mid;
                c0 = c1;
            }
            ck(cudaMemcpy(d_dest, dest.data(), dest.size() * sizeof(int), cudaMemcpyHostToDevice), "dest");
            k_chunk_scatter<<<(unsigned)nc, 1024>>>(d_chunks, d_dest, d_bin, d_ord, d_ord2);
            ck(cudaGetLastError(), "scatter");
            k_copy_back<<<(unsigned)nc, 256>>>(d_chunks, d_dest, d_ord2, d_ord);
            ck(cudaGetLastError(), "copy back");
            for (size_t j = 0; j < cur.size(); ++j) {
                const long long id = cur[j].id;
                const long long l = child(cur[j].start, mids[j]);
                const long long r = child(mids[j], cur[j].end);
                big[(size_t)id].left = l;
                big[(size_t)id].right = r;
            }
        }
        if (!small.empty()) {
            SmallJob* d_small = lvl.alloc<SmallJob>(small.size());
            ck(cudaMemcpy(d_small, small.data(), small.size() * sizeof(SmallJob), cudaMemcpyHostToDevice), "small");
            k_small<<<(unsigned)((small.size() + 63) / 64), 64>>>(d_small, (int)small.size(), d_ord, d_ord2, d_bin,
                                                                  d_tb, d_cen, d_nbox, d_nlr, d_nsc, d_flags);
            ck(cudaGetLastError(), "small nodes");
        }
        int flags = 0;
        ck(cudaMemcpy(&flags, d_flags, sizeof(int), cudaMemcpyDeviceToHost), "flags");
        if (flags) {
            if (err) *err = "a node went deeper than the small-node stack";
            return kGpuBvhUseHost;
        }
        std::vector<double> nbox(6 * 2 * (size_t)nt);
        std::vector<int> nlr(4 * (size_t)nt), nsc(4 * (size_t)nt), ord(nt);
        ck(cudaMemcpy(nbox.data(), d_nbox, nbox.size() * sizeof(double), cudaMemcpyDeviceToHost), "nodes");
        ck(cudaMemcpy(nlr.data(), d_nlr, nlr.size() * sizeof(int), cudaMemcpyDeviceToHost), "nodes");
        ck(cudaMemcpy(nsc.data(), d_nsc, nsc.size() * sizeof(int), cudaMemcpyDeviceToHost), "nodes");
        ck(cudaMemcpy(ord.data(), d_ord, ord.size() * sizeof(int), cudaMemcpyDeviceToHost), "order");

        // preorder numbering: node, left subtree, right subtree
        struct Visit { long long id; int64_t parent; int side; int depth; };
        std::vector<Visit> stack{{root, -1, 0, 1}};
        while (!stack.empty()) {
            const Visit v = stack.back();
            stack.pop_back();
            const int64_t me = (int64_t)(out.left_right.size() / 2);
            long long l, r;
            int start, count;
            if (v.id < kSmallBase) {
                const BigNode& b = big[(size_t)v.id];
                for (int k = 0; k < 3; ++k) out.bbox.push_back(b.box.lo[k]);
                for (int k = 0; k < 3; ++k) out.bbox.push_back(b.box.hi[k]);
                l = b.left; r = b.right; start = 0; count = 0;
            } else {
                const size_t slot = (size_t)(v.id - kSmallBase);
                for (int k = 0; k < 6; ++k) out.bbox.push_back(nbox[6 * slot + k]);
                l = nlr[2 * slot] < 0 ? -1 : kSmallBase + nlr[2 * slot];
                r = nlr[2 * slot + 1] < 0 ? -1 : kSmallBase + nlr[2 * slot + 1];
                start = nsc[2 * slot];
                count = nsc[2 * slot + 1];
            }
            out.left_right.push_back(-1);
            out.left_right.push_back(-1);
            out.start_count.push_back((uint32_t)start);
            out.start_count.push_back((uint32_t)count);
            if (v.parent >= 0) out.left_right[2 * (size_t)v.parent + (size_t)v.side] = (int32_t)me;
            out.max_depth = std::max(out.max_depth, v.depth);
            if (l >= 0) {
                stack.push_back(Visit{r, me, 1, v.depth + 1});
                stack.push_back(Visit{l, me, 0, v.depth + 1});
            }
        }
        out.indices.assign(ord.begin(), ord.end());
        return kGpuBvhOk;
    } catch (const CudaFail& e) {
        if (err) *err = e.what();
        cudaGetLastError();
        return kGpuBvhCudaError;
    } catch (const std::bad_alloc&) {
        if (err) *err = "device allocation failed";
        cudaGetLastError();
        return kGpuBvhCudaError;
    }
}

}  // namespace tpt
