// The octree and its interaction lists built on the GPU: the same tree, node
// numbering, source order and lists as Plan::build_tree and Plan::build_lists
// (the Stem ctor's bucketing, src/fmm/stem.cpp:3-26; Node::getNeighborGeqSize
// and getNeighborsLeqSize, src/fmm/nbor.cpp:10-644; Node::buildInteractionList,
// src/fmm/node.cpp:61-84), used when Config::device_tree is set.
//
//  1. Every source's octant digit at each level, from the same centre
//     arithmetic as the host (centre of a child = centre of the parent +
//     leng_child / 2 per axis; digit = (x > c) + 2 (y > c) + 4 (z > c)),
//     packed most significant first into a 63-bit key (21 levels).
//  2. A stable radix sort of the keys; a source's leaf level is the first
//     level whose box (the run of equal key prefixes) holds at most
//     max_node_srcs sources, or the depth cap.
//  3. The source order: a stable sort of the input order by the leaf's key
//     padded with zeros -- boxes in depth-first order, input order inside a
//     leaf (the bucketing keeps input order).
//  4. Nodes: the root and all 8 children of every split box (empty ones
//     included), sorted into depth-first pre-order (padded key, then level):
//     the host's numbering.  Parent, children, leaf flag and source range of
//     each follow from binary searches.
//  5. Lists, one thread per node: the 26 equal-or-greater neighbours, the
//     near leaves of each leaf (breadth first inside a coarser neighbour),
//     lists 2 and 4 -- counted, scanned, filled.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "plan.hpp"

namespace mlfma {
namespace {

#define TG_CK(call)                                                                        \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) return std::string("device tree: ") + #call + ": " + cudaGetErrorString(e_); \
    } while (0)

constexpr int kDepth = 21;          // octant digits in a 63-bit key
constexpr int kHardCap = 30;        // the host's depth cap
constexpr int kRsThreads = 256;
constexpr int kRsItems = 4;         // elements per thread per block
constexpr int kRsChunk = kRsThreads * kRsItems;

using u64 = unsigned long long;

// ---------------------------------------------------------------- stable radix sort
__global__ void k_rs_hist(const u64* __restrict__ keys, int n, int shift, unsigned* __restrict__ hist, int nblk) {
    __shared__ unsigned cnt[256];
    cnt[threadIdx.x] = 0;
    __syncthreads();
    for (int r = 0; r < kRsItems; ++r) {
        const int i = blockIdx.x * kRsChunk + r * kRsThreads + threadIdx.x;
        if (i < n) atomicAdd(&cnt[(keys[i] >> shift) & 255], 1u);
    }
    __syncthreads();
    hist[threadIdx.x * nblk + blockIdx.x] = cnt[threadIdx.x];
}

// exclusive scan of hist (digit-major), one block
__global__ void k_rs_scan(unsigned* __restrict__ hist, int total) {
    __shared__ unsigned part[1024];
    const int per = (total + blockDim.x - 1) / blockDim.x;
    const int i0 = threadIdx.x * per, i1 = min(total, i0 + per);
    unsigned s = 0;
    for (int i = i0; i < i1; ++i) s += hist[i];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned run = 0;
        for (int t = 0; t < static_cast<int>(blockDim.x); ++t) {
            const unsigned v = part[t];
            part[t] = run;
            run += v;
        }
    }
    __syncthreads();
    unsigned run = part[threadIdx.x];
    for (int i = i0; i < i1; ++i) {
        const unsigned v = hist[i];
        hist[i] = run;
        run += v;
    }
}

// scatter with ranks in element order: rounds of 256 elements; inside a round,
// lanes of equal digit in a warp rank by lane, warps by index
__global__ void k_rs_scatter(const u64* __restrict__ kin, const int* __restrict__ vin, int n, int shift,
                             const unsigned* __restrict__ off, int nblk, u64* __restrict__ kout, int* __restrict__ vout) {
    __shared__ unsigned running[256];
    __shared__ unsigned wcnt[kRsThreads / 32][256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    running[threadIdx.x] = 0;
    for (int r = 0; r < kRsItems; ++r) {
        for (int d = threadIdx.x; d < (kRsThreads / 32) * 256; d += kRsThreads) wcnt[d / 256][d % 256] = 0;
        __syncthreads();
        const int i = blockIdx.x * kRsChunk + r * kRsThreads + threadIdx.x;
        const bool live = i < n;
        const u64 k = live ? kin[i] : 0;
        const int d = live ? static_cast<int>((k >> shift) & 255) : 256;  // 256: no element
        const unsigned m = __match_any_sync(0xffffffffu, d);
        const unsigned wrank = __popc(m & ((1u << lane) - 1u));
        if (live && wrank == 0) wcnt[warp][d] = __popc(m);
        __syncthreads();
        if (live) {
            unsigned rank = running[d] + wrank;
            for (int w = 0; w < warp; ++w) rank += wcnt[w][d];
            const unsigned pos = off[d * nblk + blockIdx.x] + rank;
            kout[pos] = k;
            vout[pos] = vin[i];
        }
        __syncthreads();
        unsigned add = 0;
        for (int w = 0; w < kRsThreads / 32; ++w) add += wcnt[w][threadIdx.x];
        running[threadIdx.x] += add;
        __syncthreads();
    }
}

// Stable sort of (keys, vals) by key bits [0, bits); the result is in keys/vals.
std::string radix_sort(u64*& keys, int*& vals, u64*& ktmp, int*& vtmp, int n, int bits, unsigned* hist) {
    if (n <= 1) return {};
    const int nblk = (n + kRsChunk - 1) / kRsChunk;
    for (int shift = 0; shift < bits; shift += 8) {
        k_rs_hist<<<nblk, kRsThreads>>>(keys, n, shift, hist, nblk);
        k_rs_scan<<<1, 1024>>>(hist, 256 * nblk);
        k_rs_scatter<<<nblk, kRsThreads>>>(keys, vals, n, shift, hist, nblk, ktmp, vtmp);
        TG_CK(cudaGetLastError());
        std::swap(keys, ktmp);
        std::swap(vals, vtmp);
    }
    return {};
}

// ---------------------------------------------------------------- tree
__global__ void k_digits(const double* __restrict__ centers, int n, double root_leng, u64* __restrict__ key,
                         int* __restrict__ idx) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const double x[3] = {centers[3 * s], centers[3 * s + 1], centers[3 * s + 2]};
    double c[3] = {0.0, 0.0, 0.0}, leng = root_leng;
    u64 k = 0;
    for (int l = 0; l < kDepth; ++l) {
        const int b = (x[0] > c[0]) + 2 * (x[1] > c[1]) + 4 * (x[2] > c[2]);
        k = (k << 3) | static_cast<u64>(b);
        const double lc = leng / 2.0;
        for (int a = 0; a < 3; ++a) c[a] = c[a] + lc / 2.0 * (((b >> a) & 1) ? 1.0 : -1.0);
        leng = lc;
    }
    key[s] = k;
    idx[s] = s;
}

__device__ __forceinline__ u64 prefix_of(u64 k, int l) { return l == 0 ? 0 : k >> (3 * (kDepth - l)); }

// first position in sorted[0, n) whose level-l prefix is >= p
__device__ int lower_prefix(const u64* sorted, int n, int l, u64 p) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (prefix_of(sorted[mid], l) < p) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// leaf level of the source at sorted position i (depth overflow: *err = 1)
__global__ void k_leaf_level(const u64* __restrict__ sk, const int* __restrict__ sv, int n, int mns, int max_level,
                             int* __restrict__ leaf_of_src, int* __restrict__ err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const u64 k = sk[i];
    int L = -1;
    for (int l = 0; l <= kDepth; ++l) {
        const u64 p = prefix_of(k, l);
        const int cnt = lower_prefix(sk, n, l, p + 1) - lower_prefix(sk, n, l, p);
        const bool split = cnt > mns && (max_level <= 0 || l < max_level) && l < kHardCap;
        if (!split) { L = l; break; }
        if (l == kDepth) break;
    }
    if (L < 0 || L > kDepth) {
        atomicExch(err, 1);
        L = kDepth;
    }
    leaf_of_src[sv[i]] = L;
}

__global__ void k_padded(const u64* __restrict__ key, const int* __restrict__ leaf_of_src, int n, u64* __restrict__ pk,
                         int* __restrict__ idx) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int sh = 3 * (kDepth - leaf_of_src[s]);
    pk[s] = sh >= 64 ? 0 : (key[s] >> sh) << sh;
    idx[s] = s;
}

// split boxes: at sorted position i, every level l below its leaf level where
// i starts a run of equal prefixes; count pass (out == nullptr) or fill
__global__ void k_splits(const u64* __restrict__ sk, const int* __restrict__ sv, int n,
                         const int* __restrict__ leaf_of_src, const int* __restrict__ base, int* __restrict__ count,
                         u64* __restrict__ out_pk, int* __restrict__ out_lv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int L = leaf_of_src[sv[i]];
    int c = 0;
    for (int l = 0; l < L; ++l) {
        const bool start = i == 0 || prefix_of(sk[i - 1], l) != prefix_of(sk[i], l);
        if (!start) continue;
        if (out_pk) {
            // children of the split box (l, p): (l + 1, 8 p + b)
            const u64 p = prefix_of(sk[i], l);
            for (int b = 0; b < 8; ++b) {
                const int at = 1 + 8 * (base[i] + c) + b;
                const u64 cp = p * 8 + static_cast<u64>(b);
                out_pk[at] = l + 1 == kDepth ? cp : cp << (3 * (kDepth - l - 1));
                out_lv[at] = l + 1;
            }
        }
        ++c;
    }
    if (!out_pk) count[i] = c;
}

// exclusive scan of a[0, n) in place, one block of 1024 threads; *total = sum
__global__ void k_scan_int(int* __restrict__ a, int n, int* __restrict__ total) {
    __shared__ long long part[1024];
    const int per = (n + blockDim.x - 1) / blockDim.x;
    const int i0 = min(n, static_cast<int>(threadIdx.x) * per), i1 = min(n, i0 + per);
    long long s = 0;
    for (int i = i0; i < i1; ++i) s += a[i];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long run = 0;
        for (int t = 0; t < static_cast<int>(blockDim.x); ++t) {
            const long long v = part[t];
            part[t] = run;
            run += v;
        }
        *total = run > 0x7fffffffLL ? -1 : static_cast<int>(run);
    }
    __syncthreads();
    long long run = part[threadIdx.x];
    for (int i = i0; i < i1; ++i) {
        const int v = a[i];
        a[i] = static_cast<int>(run);
        run += v;
    }
}

// node records in depth-first order (padded key pk[id], level lv[id])
__device__ int find_node(const u64* pk, const int* lv, int nn, u64 key, int level) {
    int lo = 0, hi = nn;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (pk[mid] < key) lo = mid + 1; else hi = mid;
    }
    for (int j = lo; j < nn && pk[j] == key; ++j)
        if (lv[j] == level) return j;
    return -1;
}

__global__ void k_nodes(const u64* __restrict__ pk, const int* __restrict__ lv, int nn, const u64* __restrict__ sk,
                        int n, const u64* __restrict__ perm_pk, int* __restrict__ parent, int* __restrict__ branch,
                        int* __restrict__ child, int* __restrict__ leaf, int* __restrict__ sbeg,
                        int* __restrict__ scnt) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= nn) return;
    const int l = lv[id];
    const u64 key = pk[id];
    const u64 p = l == 0 ? 0 : key >> (3 * (kDepth - l));
    // sources in the box: keys with this prefix; their first tree-order position
    const int lo = lower_prefix(sk, n, l, p);
    scnt[id] = lower_prefix(sk, n, l, p + 1) - lo;
    int a = 0, b2 = n;
    while (a < b2) {
        const int mid = (a + b2) >> 1;
        if (perm_pk[mid] < key) a = mid + 1; else b2 = mid;
    }
    sbeg[id] = a;
    if (l == 0) {
        parent[id] = -1;
        branch[id] = 0;
        return;
    }
    const int br = static_cast<int>(p & 7);
    const u64 pp = p >> 3;
    const u64 ppk = l - 1 == 0 ? 0 : pp << (3 * (kDepth - l + 1));
    const int par = find_node(pk, lv, nn, ppk, l - 1);
    parent[id] = par;
    branch[id] = br;
    if (par >= 0) {
        child[par * 8 + br] = id;
        leaf[par] = 0;
    }
}

// ---------------------------------------------------------------- lists
__constant__ int c_dirs[26][3];

// Node::getNeighborGeqSize (per axis; the host's nbr_geq)
__device__ int nbr_geq_d(const int* parent, const int* branch, const int* child, const int* leaf, int id, int dx,
                         int dy, int dz) {
    // iterative form of the recursion: walk up while the direction leaves the
    // parent, remembering each level's (target, all_out), then walk down
    int tgt[kHardCap + 1];
    bool allo[kHardCap + 1];
    int depth = 0;
    int cur = id;
    int d[3] = {dx, dy, dz};
    while (true) {
        if (parent[cur] < 0) return -1;
        const int b = branch[cur];
        int dout[3] = {0, 0, 0}, mask = 0;
        bool any_out = false, all_out = true;
        for (int a = 0; a < 3; ++a) {
            if (!d[a]) continue;
            mask |= 1 << a;
            const int ba = (b >> a) & 1;
            const bool out = (d[a] > 0 && ba == 1) || (d[a] < 0 && ba == 0);
            if (out) { dout[a] = d[a]; any_out = true; } else { all_out = false; }
        }
        const int target = b ^ mask;
        if (!any_out) {
            int nb = child[parent[cur] * 8 + target];
            // unwind
            for (int k = depth - 1; k >= 0; --k) {
                if (nb < 0) return -1;
                if (leaf[nb]) nb = allo[k] ? nb : -1;
                else nb = child[nb * 8 + tgt[k]];
            }
            return nb;
        }
        if (depth > kHardCap) return -1;
        tgt[depth] = target;
        allo[depth] = all_out;
        ++depth;
        cur = parent[cur];
        d[0] = dout[0];
        d[1] = dout[1];
        d[2] = dout[2];
    }
}

__global__ void k_nbors(int nn, const int* parent, const int* branch, const int* child, const int* leaf,
                        int* __restrict__ nb26) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= nn) return;
    for (int i = 0; i < 26; ++i)
        nb26[id * 26 + i] = parent[id] < 0 ? -1 : nbr_geq_d(parent, branch, child, leaf, id, c_dirs[i][0], c_dirs[i][1],
                                                            c_dirs[i][2]);
}

// near leaves of leaf id (Node::getNeighborsLeqSize), count or fill.  The
// host's breadth-first queue emits the leaves inside a neighbour by depth and,
// at one depth, in child-index path order; a depth-limited walk per depth
// gives the same order with a stack of the tree's height.
__global__ void k_near(int nn, const int* child, const int* leaf, const int* nb26, const int* base, int* count,
                       int* out) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= nn) return;
    if (!leaf[id]) {
        if (!out) count[id] = 0;
        return;
    }
    int stk[kHardCap + 1], nxt[kHardCap + 1];
    int c = 0;
    for (int i = 0; i < 26; ++i) {
        const int nb = nb26[id * 26 + i];
        if (nb < 0) continue;
        const int* d = c_dirs[i];
        for (int depth = 0; depth <= kHardCap; ++depth) {
            bool deeper = false;
            int top = 0;
            stk[0] = nb;
            nxt[0] = -1;
            while (top >= 0) {
                const int cur = stk[top];
                if (nxt[top] < 0) {  // first visit
                    if (top == depth) {
                        if (leaf[cur]) {
                            if (out) out[base[id] + c] = cur;
                            ++c;
                        } else {
                            deeper = true;
                        }
                        --top;
                        continue;
                    }
                    if (leaf[cur]) {  // emitted at its own depth
                        --top;
                        continue;
                    }
                    nxt[top] = 0;
                }
                int cc = nxt[top];
                for (; cc < 8; ++cc) {  // children on the face, edge or corner toward the box
                    bool ok = true;
                    for (int a = 0; a < 3; ++a) {
                        const int ca = (cc >> a) & 1;
                        if ((d[a] > 0 && ca != 0) || (d[a] < 0 && ca != 1)) ok = false;
                    }
                    if (ok) break;
                }
                if (cc >= 8) {
                    --top;
                    continue;
                }
                nxt[top] = cc + 1;
                const int nx = child[cur * 8 + cc];
                if (nx < 0) continue;  // not reached: a split box has all 8 children
                ++top;
                stk[top] = nx;
                nxt[top] = -1;
            }
            if (!deeper) break;
        }
    }
    if (!out) count[id] = c;
}

// lists 2 and 4 of node id (Node::buildInteractionList), count or fill
__global__ void k_ilists(int nn, const int* parent, const int* child, const int* leaf, const int* scnt,
                         const int* nb26, const int* base2, const int* base4, int* cnt2, int* cnt4, int* out2,
                         int* out4) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= nn) return;
    int c2 = 0, c4 = 0;
    const int par = parent[id];
    if (par >= 0) {
        auto contains = [&](int v) {
            for (int i = 0; i < 26; ++i)
                if (nb26[id * 26 + i] == v) return true;
            return false;
        };
        for (int i = 0; i < 26; ++i) {
            const int bn = nb26[par * 26 + i];
            if (bn < 0 || scnt[bn] == 0) continue;
            if (leaf[bn]) {
                if (!contains(bn)) {
                    if (out4) out4[base4[id] + c4] = bn;
                    ++c4;
                }
                continue;
            }
            for (int c = 0; c < 8; ++c) {
                const int ch = child[bn * 8 + c];
                if (ch >= 0 && !contains(ch) && scnt[ch] > 0) {
                    if (out2) out2[base2[id] + c2] = ch;
                    ++c2;
                }
            }
        }
    }
    if (!out2) {
        cnt2[id] = c2;
        cnt4[id] = c4;
    }
}

template <class T>
struct DevBuf {
    T* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
    cudaError_t alloc(size_t n) { return cudaMalloc(&p, sizeof(T) * std::max<size_t>(n, 1)); }
};

std::string scan_counts(int* d, int n, int* total_h) {
    DevBuf<int> tot;
    TG_CK(tot.alloc(1));
    k_scan_int<<<1, 1024>>>(d, n, tot.p);
    TG_CK(cudaMemcpy(total_h, tot.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (*total_h < 0) return "device tree: more than 2^31 list entries";
    return {};
}

}  // namespace

std::string build_tree_lists_device(Plan& P, const std::vector<double>& centers) {
    const int n = P.n;
    const Config& cfg = P.cfg;
    if (n < 2) return "host: fewer than two sources";
    const int T = 256;
    auto blocks = [&](long long m) { return static_cast<int>((m + T - 1) / T); };
    DevBuf<double> d_c;
    DevBuf<u64> k0, k1, skeep;
    DevBuf<int> v0, v1, leafL, err;
    DevBuf<unsigned> hist;
    TG_CK(d_c.alloc(3 * static_cast<size_t>(n)));
    TG_CK(cudaMemcpy(d_c.p, centers.data(), sizeof(double) * 3 * n, cudaMemcpyHostToDevice));
    TG_CK(k0.alloc(n));
    TG_CK(k1.alloc(n));
    TG_CK(skeep.alloc(n));
    TG_CK(v0.alloc(n));
    TG_CK(v1.alloc(n));
    TG_CK(leafL.alloc(n));
    TG_CK(err.alloc(1));
    TG_CK(cudaMemset(err.p, 0, sizeof(int)));
    const int nblk = (n + kRsChunk - 1) / kRsChunk;
    TG_CK(hist.alloc(static_cast<size_t>(256) * std::max(nblk, 1)));
    // 1-2: keys, sorted keys, leaf levels
    k_digits<<<blocks(n), T>>>(d_c.p, n, cfg.root_leng, k0.p, v0.p);
    TG_CK(cudaMemcpy(skeep.p, k0.p, sizeof(u64) * n, cudaMemcpyDeviceToDevice));  // keys in input order
    u64 *ka = k0.p, *kb = k1.p;
    int *va = v0.p, *vb = v1.p;
    std::string e = radix_sort(ka, va, kb, vb, n, 3 * kDepth, hist.p);
    if (!e.empty()) return e;
    k_leaf_level<<<blocks(n), T>>>(ka, va, n, cfg.max_node_srcs, cfg.max_level, leafL.p, err.p);
    {
        int herr = 0;
        TG_CK(cudaMemcpy(&herr, err.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (herr) return "host: the tree is deeper than the 21 levels of the device keys";
    }
    // split boxes and the node records
    DevBuf<int> scount;
    TG_CK(scount.alloc(n));
    k_splits<<<blocks(n), T>>>(ka, va, n, leafL.p, nullptr, scount.p, nullptr, nullptr);
    int nsplit = 0;
    e = scan_counts(scount.p, n, &nsplit);
    if (!e.empty()) return e;
    const int nn = 1 + 8 * nsplit;
    DevBuf<u64> npk, npk2;
    DevBuf<int> nlv, nlv2;
    TG_CK(npk.alloc(nn));
    TG_CK(npk2.alloc(nn));
    TG_CK(nlv.alloc(nn));
    TG_CK(nlv2.alloc(nn));
    TG_CK(cudaMemset(npk.p, 0, sizeof(u64)));  // the root: key 0, level 0
    TG_CK(cudaMemset(nlv.p, 0, sizeof(int)));
    k_splits<<<blocks(n), T>>>(ka, va, n, leafL.p, scount.p, nullptr, npk.p, nlv.p);
    // 3: the source order (stable by padded leaf key over the input order)
    DevBuf<u64> ppk;
    TG_CK(ppk.alloc(n));
    DevBuf<int> pidx;
    TG_CK(pidx.alloc(n));
    k_padded<<<blocks(n), T>>>(skeep.p, leafL.p, n, ppk.p, pidx.p);
    u64* pa = ppk.p;
    int* pv = pidx.p;
    u64* pb = kb;  // scratch of the key sort is free now
    int* pw = vb;
    e = radix_sort(pa, pv, pb, pw, n, 3 * kDepth, hist.p);
    if (!e.empty()) return e;
    // 4: nodes in depth-first pre-order: stable by level, then by padded key
    DevBuf<int> nidx, nidx2;
    TG_CK(nidx.alloc(nn));
    TG_CK(nidx2.alloc(nn));
    {
        std::vector<int> iota(nn);
        for (int i = 0; i < nn; ++i) iota[i] = i;
        TG_CK(cudaMemcpy(nidx.p, iota.data(), sizeof(int) * nn, cudaMemcpyHostToDevice));
    }
    // level as the first (less significant) key: keys = level, values = record index
    DevBuf<u64> lvk, lvk2;
    TG_CK(lvk.alloc(nn));
    TG_CK(lvk2.alloc(nn));
    {
        std::vector<int> hl(nn);
        TG_CK(cudaMemcpy(hl.data(), nlv.p, sizeof(int) * nn, cudaMemcpyDeviceToHost));
        std::vector<u64> hk(hl.begin(), hl.end());
        TG_CK(cudaMemcpy(lvk.p, hk.data(), sizeof(u64) * nn, cudaMemcpyHostToDevice));
    }
    DevBuf<unsigned> nhist;
    const int nblk2 = (nn + kRsChunk - 1) / kRsChunk;
    TG_CK(nhist.alloc(static_cast<size_t>(256) * std::max(nblk2, 1)));
    u64 *la = lvk.p, *lb = lvk2.p;
    int *ia = nidx.p, *ib = nidx2.p;
    e = radix_sort(la, ia, lb, ib, nn, 8, nhist.p);
    if (!e.empty()) return e;
    std::vector<int> order1(nn);
    TG_CK(cudaMemcpy(order1.data(), ia, sizeof(int) * nn, cudaMemcpyDeviceToHost));
    std::vector<u64> hpk(nn);
    std::vector<int> hlv(nn);
    TG_CK(cudaMemcpy(hpk.data(), npk.p, sizeof(u64) * nn, cudaMemcpyDeviceToHost));
    TG_CK(cudaMemcpy(hlv.data(), nlv.p, sizeof(int) * nn, cudaMemcpyDeviceToHost));
    {
        std::vector<u64> k2(nn);
        for (int i = 0; i < nn; ++i) k2[i] = hpk[order1[i]];
        TG_CK(cudaMemcpy(lvk.p, k2.data(), sizeof(u64) * nn, cudaMemcpyHostToDevice));
        TG_CK(cudaMemcpy(nidx.p, order1.data(), sizeof(int) * nn, cudaMemcpyHostToDevice));
    }
    la = lvk.p;
    lb = lvk2.p;
    ia = nidx.p;
    ib = nidx2.p;
    e = radix_sort(la, ia, lb, ib, nn, 3 * kDepth, nhist.p);
    if (!e.empty()) return e;
    std::vector<int> order(nn);
    TG_CK(cudaMemcpy(order.data(), ia, sizeof(int) * nn, cudaMemcpyDeviceToHost));
    std::vector<u64> spk(nn);
    std::vector<int> slv(nn);
    for (int i = 0; i < nn; ++i) {
        spk[i] = hpk[order[i]];
        slv[i] = hlv[order[i]];
    }
    TG_CK(cudaMemcpy(npk2.p, spk.data(), sizeof(u64) * nn, cudaMemcpyHostToDevice));
    TG_CK(cudaMemcpy(nlv2.p, slv.data(), sizeof(int) * nn, cudaMemcpyHostToDevice));
    DevBuf<int> par, br, ch, lf, sb, sc;
    TG_CK(par.alloc(nn));
    TG_CK(br.alloc(nn));
    TG_CK(ch.alloc(8 * static_cast<size_t>(nn)));
    TG_CK(lf.alloc(nn));
    TG_CK(sb.alloc(nn));
    TG_CK(sc.alloc(nn));
    TG_CK(cudaMemset(ch.p, 0xff, sizeof(int) * 8 * nn));
    {
        std::vector<int> ones(nn, 1);
        TG_CK(cudaMemcpy(lf.p, ones.data(), sizeof(int) * nn, cudaMemcpyHostToDevice));
    }
    k_nodes<<<blocks(nn), T>>>(npk2.p, nlv2.p, nn, ka, n, pa, par.p, br.p, ch.p, lf.p, sb.p, sc.p);
    // 5: lists
    TG_CK(cudaMemcpyToSymbol(c_dirs, plan_directions(), sizeof(int) * 26 * 3));
    DevBuf<int> nb26;
    TG_CK(nb26.alloc(26 * static_cast<size_t>(nn)));
    k_nbors<<<blocks(nn), T>>>(nn, par.p, br.p, ch.p, lf.p, nb26.p);
    DevBuf<int> ncnt, c2, c4;
    TG_CK(ncnt.alloc(nn));
    TG_CK(c2.alloc(nn));
    TG_CK(c4.alloc(nn));
    k_near<<<blocks(nn), T>>>(nn, ch.p, lf.p, nb26.p, nullptr, ncnt.p, nullptr);
    k_ilists<<<blocks(nn), T>>>(nn, par.p, ch.p, lf.p, sc.p, nb26.p, nullptr, nullptr, c2.p, c4.p, nullptr, nullptr);
    int nnear = 0, n2 = 0, n4 = 0;
    if (!(e = scan_counts(ncnt.p, nn, &nnear)).empty() || !(e = scan_counts(c2.p, nn, &n2)).empty() ||
        !(e = scan_counts(c4.p, nn, &n4)).empty())
        return e;
    DevBuf<int> onear, o2, o4;
    TG_CK(onear.alloc(nnear));
    TG_CK(o2.alloc(n2));
    TG_CK(o4.alloc(n4));
    k_near<<<blocks(nn), T>>>(nn, ch.p, lf.p, nb26.p, ncnt.p, nullptr, onear.p);
    k_ilists<<<blocks(nn), T>>>(nn, par.p, ch.p, lf.p, sc.p, nb26.p, c2.p, c4.p, nullptr, nullptr, o2.p, o4.p);
    TG_CK(cudaGetLastError());
    // back to the host plan
    std::vector<int> hpar(nn), hbr(nn), hch(8 * static_cast<size_t>(nn)), hlf(nn), hsb(nn), hsc(nn),
        hnb(26 * static_cast<size_t>(nn)), hnc(nn), hc2(nn), hc4(nn), hnear(nnear), h2(n2), h4(n4), hperm(n);
    TG_CK(cudaMemcpy(hpar.data(), par.p, sizeof(int) * nn, cudaMemcpyDeviceToHost));
    TG_CK(cudaMemcpy(hbr.data(), br.p, sizeof(int) * nn, cudaMemcpyDeviceToHost));
    TG_CK(cudaMemcpy(hch.data(), ch.p, sizeof(int) * 8 * nn, cudaMemcpyDeviceToHost));
    TG_CK(cudaMemcpy(hlf.data(), lf.p, sizeof(int) * nn, cudaMemcpyDeviceToHost));
    TG_CK(cudaMemcpy(hsb.data(), sb.p, sizeof(int) * nn, cudaMemcpyDeviceToHost));
    TG_CK(cudaMemcpy(hsc.data(), sc.p, sizeof(int) * nn, cudaMemcpyDeviceToHost));
    TG_CK(cudaMemcpy(hnb.data(), nb26.p, sizeof(int) * 26 * nn, cudaMemcpyDeviceToHost));
    TG_CK(cudaMemcpy(hnc.data(), ncnt.p, sizeof(int) * nn, cudaMemcpyDeviceToHost));
    TG_CK(cudaMemcpy(hc2.data(), c2.p, sizeof(int) * nn, cudaMemcpyDeviceToHost));
    TG_CK(cudaMemcpy(hc4.data(), c4.p, sizeof(int) * nn, cudaMemcpyDeviceToHost));
    if (nnear) TG_CK(cudaMemcpy(hnear.data(), onear.p, sizeof(int) * nnear, cudaMemcpyDeviceToHost));
    if (n2) TG_CK(cudaMemcpy(h2.data(), o2.p, sizeof(int) * n2, cudaMemcpyDeviceToHost));
    if (n4) TG_CK(cudaMemcpy(h4.data(), o4.p, sizeof(int) * n4, cudaMemcpyDeviceToHost));
    TG_CK(cudaMemcpy(hperm.data(), pv, sizeof(int) * n, cudaMemcpyDeviceToHost));
    P.nodes.assign(nn, Node{});
    P.perm = hperm;
    P.leaves.clear();
    P.max_level = 0;
    P.n_list2 = P.n_list4 = 0;
    for (int id = 0; id < nn; ++id) {
        Node& nd = P.nodes[id];
        nd.level = slv[id];
        nd.parent = hpar[id];
        nd.branch = hbr[id];
        for (int b = 0; b < 8; ++b) nd.child[b] = hch[8 * static_cast<size_t>(id) + b];
        nd.leaf = hlf[id] != 0;
        nd.src_begin = hsb[id];
        nd.src_count = hsc[id];
        if (nd.parent < 0) {
            nd.leng = cfg.root_leng;
        } else {  // the host's geometry (Plan::build_tree); parents come first in pre-order
            const Node& Pn = P.nodes[nd.parent];
            nd.leng = Pn.leng / 2.0;
            const double pm[3] = {(nd.branch & 1) ? 1.0 : -1.0, (nd.branch & 2) ? 1.0 : -1.0,
                                  (nd.branch & 4) ? 1.0 : -1.0};
            for (int k = 0; k < 3; ++k) nd.center[k] = Pn.center[k] + nd.leng / 2.0 * pm[k];
            nd.ix = 2 * Pn.ix + (nd.branch & 1);
            nd.iy = 2 * Pn.iy + ((nd.branch >> 1) & 1);
            nd.iz = 2 * Pn.iz + ((nd.branch >> 2) & 1);
        }
        for (int i = 0; i < 26; ++i)
            if (hnb[26 * static_cast<size_t>(id) + i] >= 0) nd.nbors.push_back(hnb[26 * static_cast<size_t>(id) + i]);
        const int ne = (id + 1 < nn ? hnc[id + 1] : nnear) - hnc[id];
        nd.near_nbors.assign(hnear.begin() + hnc[id], hnear.begin() + hnc[id] + ne);
        const int e2 = (id + 1 < nn ? hc2[id + 1] : n2) - hc2[id];
        nd.ilist.assign(h2.begin() + hc2[id], h2.begin() + hc2[id] + e2);
        const int e4 = (id + 1 < nn ? hc4[id + 1] : n4) - hc4[id];
        nd.leaf_ilist.assign(h4.begin() + hc4[id], h4.begin() + hc4[id] + e4);
        P.n_list2 += e2;
        P.n_list4 += e4;
        if (nd.leaf) {
            P.leaves.push_back(id);
            P.max_level = std::max(P.max_level, nd.level);
        }
    }
    P.src_center.resize(3 * static_cast<size_t>(n));
    for (int t = 0; t < n; ++t)
        for (int k = 0; k < 3; ++k) P.src_center[3 * t + k] = centers[3 * P.perm[t] + k];
    return {};
}

}  // namespace mlfma
