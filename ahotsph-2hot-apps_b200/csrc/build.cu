// build.cu -- the tree build and the MAC walk on the GPU: the producer side
// of the batched lists (nlnhost.h's nln_tree_build + nln_tree_walk) without
// leaving the device.
//
// Every step follows the host builder and shares its arithmetic
// (host/tree_math.h), and this file is compiled without fused
// multiply-adds (-fmad=false) as the host library is without contraction,
// so the tables and lists are bit-identical to the host's:
//   bounding cube     exact min / max of the FP32 positions, enlarged on the host as nlnhost.cpp
//   Morton keys       21 bits per axis, stable radix sort of (key, input index)
//   cells             level-synchronous octant splits of the sorted keys, one level per pass
//   moments           FP64 sums over each cell's bodies in the canonical blocked order of
//                     nlnhost.cpp (64 bodies, 64 partials, then in order): one thread per
//                     block at each of the three levels
//   tables, rcrit     nln_cell_tables, nln_cell_rcrit (tree_math.h), one thread per cell
//   sink groups       the runs of nlnhost.cpp's collect_groups: small children of every
//                     large cell merged in order, sorted by first body
//   walk              nln_walk_group (tree_math.h), one thread per group: a counting pass,
//                     offsets, a filling pass
// Algorithms restated from the reference: nln/cofm.c:96-231,247-574 (moments,
// critical radii), nln/mac.c:1774-1844 (DLRcritMAC), nln/mac.c:91-111 (images).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cub/cub.cuh>
#include <vector>

#include "build.cuh"
#include "common.cuh"
#include "host/tree_math.h"

namespace {

constexpr int KEY_LEVELS = 21;
constexpr int kSumBlock = 64;  // the canonical sum's block (nlnhost.cpp)
constexpr int kThreads = 256;

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

__host__ __device__ inline uint64_t spread3(uint32_t v) {
    uint64_t x = v & 0x1fffff;
    x = (x | x << 32) & 0x1f00000000ffffULL;
    x = (x | x << 16) & 0x1f0000ff0000ffULL;
    x = (x | x << 8) & 0x100f00f00f00f00fULL;
    x = (x | x << 4) & 0x10c30c30c30c30c3ULL;
    x = (x | x << 2) & 0x1249249249249249ULL;
    return x;
}

unsigned grid_of(int64_t n, int threads = kThreads) {
    return (unsigned)std::max<int64_t>(1, (n + threads - 1) / threads);
}

// device buffers freed at the end of the build unless released to the
// caller; from a memory pool (stream-ordered on st) when one is given
struct Bufs {
    cudaMemPool_t pool = nullptr;
    cudaStream_t st = nullptr;
    std::vector<void *> held;
    ~Bufs() {
        for (void *p : held) free_one(p);
    }
    void free_one(void *p) {
        if (pool)
            cudaFreeAsync(p, st);
        else
            cudaFree(p);
    }
    template <typename T>
    cudaError_t get(T **p, size_t n) {
        *p = nullptr;
        const size_t bytes = std::max<size_t>(1, n) * sizeof(T);
        cudaError_t e = pool ? cudaMallocFromPoolAsync((void **)p, bytes, pool, st)
                             : cudaMalloc((void **)p, bytes);
        if (e == cudaSuccess)
            held.push_back(*p);
        return e;
    }
    template <typename T>
    void release(T *p) {  // ownership passes on
        auto it = std::find(held.begin(), held.end(), (void *)p);
        if (it != held.end())
            held.erase(it);
    }
    template <typename T>
    void drop(T *p) {
        auto it = std::find(held.begin(), held.end(), (void *)p);
        if (it != held.end()) {
            free_one(*it);
            held.erase(it);
        }
    }
};

#define BC(call)                                                       \
    do {                                                               \
        cudaError_t _e = (call);                                       \
        if (_e != cudaSuccess)                                         \
            return gc::cuda_status(_e, "GPU tree build: " #call);     \
    } while (0)

// ------------------------------------------------------------ bounding cube
// Per-block min / max of the positions; a non-finite position, or with
// box > 0 one outside [0, box), sets *bad.
__global__ void k_bbox(const float4 *__restrict__ b, int64_t n, double box, float *blo, float *bhi,
                       unsigned *bad) {
    __shared__ float slo[3][kThreads], shi[3][kThreads];
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    unsigned flag = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float4 p = b[i];
        const float x[3] = {p.x, p.y, p.z};
        for (int d = 0; d < 3; d++) {
            if (!isfinite(x[d]) || (box > 0 && !(x[d] >= 0.0f && (double)x[d] < box)))
                flag = 1;
            lo[d] = fminf(lo[d], x[d]);
            hi[d] = fmaxf(hi[d], x[d]);
        }
    }
    if (flag)
        atomicOr(bad, 1u);
    for (int d = 0; d < 3; d++) {
        slo[d][threadIdx.x] = lo[d];
        shi[d][threadIdx.x] = hi[d];
    }
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int d = 0; d < 3; d++) {
                slo[d][threadIdx.x] = fminf(slo[d][threadIdx.x], slo[d][threadIdx.x + w]);
                shi[d][threadIdx.x] = fmaxf(shi[d][threadIdx.x], shi[d][threadIdx.x + w]);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int d = 0; d < 3; d++) {
            blo[3 * blockIdx.x + d] = slo[d][0];
            bhi[3 * blockIdx.x + d] = shi[d][0];
        }
}

// ------------------------------------------------------------ keys, sort, permute
__global__ void k_keys(const float4 *__restrict__ b, int64_t n, double ox, double oy, double oz,
                       double scale, uint64_t *key, int64_t *idx) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float4 p = b[i];
    const double x[3] = {p.x, p.y, p.z}, o[3] = {ox, oy, oz};
    uint32_t c[3];
    for (int d = 0; d < 3; d++) {
        const double u = (x[d] - o[d]) * scale;
        int64_t v = (int64_t)floor(u);
        v = v < 0 ? 0 : (v > (1 << KEY_LEVELS) - 1 ? (1 << KEY_LEVELS) - 1 : v);
        c[d] = (uint32_t)v;
    }
    key[i] = spread3(c[0]) << 2 | spread3(c[1]) << 1 | spread3(c[2]);
    idx[i] = i;
}

__global__ void k_permute(const float4 *__restrict__ b, const int64_t *__restrict__ order,
                          int64_t n, float *spos, float *smass, float4 *points) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float4 p = b[order[i]];
    spos[3 * i] = p.x;
    spos[3 * i + 1] = p.y;
    spos[3 * i + 2] = p.z;
    smass[i] = p.w;
    points[i] = p;
}

// ------------------------------------------------------------ cells
struct Cells {
    int64_t *first;
    int32_t *count, *child, *nchild, *level;
    double *gc;    // 3 per cell
    double *side;
};

// Frontier cells [lo, lo + nf): children per octant by binary search of the
// sorted keys (nlnhost.cpp build_cells); nk[f] their number, bounds[9 f ..]
// the octants' first bodies.
__global__ void k_split_count(Cells C, int64_t lo, int64_t nf, const uint64_t *__restrict__ keys,
                              int leaf_max, int64_t *nk, int64_t *bounds) {
    const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf)
        return;
    const int64_t c = lo + f;
    nk[f] = 0;
    const int32_t cnt = C.count[c], lev = C.level[c];
    if (cnt <= leaf_max || lev >= KEY_LEVELS)
        return;
    const int shift = 3 * (KEY_LEVELS - 1 - lev);
    int64_t a0 = C.first[c], hi = C.first[c] + cnt;
    bounds[f * 9] = a0;
    int k = 0;
    for (int o = 0; o < 8; o++) {
        int64_t a = a0, bb = hi;
        while (a < bb) {
            const int64_t mid = (a + bb) / 2;
            if ((int)((keys[mid] >> shift) & 7) <= o)
                a = mid + 1;
            else
                bb = mid;
        }
        bounds[f * 9 + o + 1] = a;
        if (a > a0)
            k++;
        a0 = a;
    }
    nk[f] = k;
}

// Write the children of frontier cell f at base + off[f] .. in octant order.
__global__ void k_split_write(Cells C, int64_t lo, int64_t nf, const int64_t *__restrict__ nk,
                              const int64_t *__restrict__ bounds, const int64_t *__restrict__ off,
                              int64_t base) {
    const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf || nk[f] == 0)
        return;
    const int64_t c = lo + f;
    C.child[c] = (int32_t)(base + off[f]);
    C.nchild[c] = (int32_t)nk[f];
    const double side = C.side[c];
    int k = 0;
    for (int o = 0; o < 8; o++) {
        const int64_t a = bounds[f * 9 + o], b = bounds[f * 9 + o + 1];
        if (b <= a)
            continue;
        const int64_t d = base + off[f] + k;
        C.first[d] = a;
        C.count[d] = (int32_t)(b - a);
        C.child[d] = -1;
        C.nchild[d] = 0;
        C.level[d] = C.level[c] + 1;
        C.side[d] = 0.5 * side;
        C.gc[3 * d] = C.gc[3 * c] + ((o >> 2) & 1 ? 0.25 : -0.25) * side;
        C.gc[3 * d + 1] = C.gc[3 * c + 1] + ((o >> 1) & 1 ? 0.25 : -0.25) * side;
        C.gc[3 * d + 2] = C.gc[3 * c + 2] + ((o >> 0) & 1 ? 0.25 : -0.25) * side;
        k++;
    }
}

// ------------------------------------------------------------ canonical sums
// Pass 1 (K = 4): mass and offset sums about the geometric centre; pass 2
// (K = NLN_NMOM, + 1 max): raw moments about the centre of mass.  Level 0:
// one thread per block of 64 bodies of a cell; level 1: per block of 64
// level-0 partials; level 2: per cell, its level-1 partials in order.
template <int K>
__device__ inline void body_terms(const float *spos, const float *smass, int64_t b,
                                  const double *ctr, double *a, double &mx) {
    if (K == 4)
        nln_mass_terms(spos + 3 * b, smass[b], ctr, a);
    else
        mx = fmax(mx, nln_moment_terms(spos + 3 * b, smass[b], ctr, a));
}

__device__ inline int64_t owner(const int64_t *off, int64_t ncells, int64_t j) {
    int64_t a = 0, b = ncells;  // the last cell c with off[c] <= j
    while (b - a > 1) {
        const int64_t mid = (a + b) / 2;
        if (off[mid] <= j)
            a = mid;
        else
            b = mid;
    }
    return a;
}

template <int K>
__global__ void k_sum0(const Cells C, int64_t ncells, const int64_t *__restrict__ o0,
                       int64_t total, const float *spos, const float *smass, const double *ctr,
                       double *p0) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= total)
        return;
    const int64_t c = owner(o0, ncells, j);
    const int64_t blk = j - o0[c];
    const int64_t first = C.first[c], cnt = C.count[c];
    const double cc[3] = {ctr[3 * c], ctr[3 * c + 1], ctr[3 * c + 2]};
    double a[K + 1];
    for (int q = 0; q <= K; q++) a[q] = 0.0;
    double mx = 0.0;
    const int64_t k1 = cnt < (blk + 1) * kSumBlock ? cnt : (blk + 1) * kSumBlock;
    for (int64_t k = blk * kSumBlock; k < k1; k++) body_terms<K>(spos, smass, first + k, cc, a, mx);
    a[K] = mx;
    for (int q = 0; q <= K; q++) p0[j * (K + 1) + q] = a[q];
}

template <int K>
__global__ void k_sum1(const Cells C, int64_t ncells, const int64_t *__restrict__ o0,
                       const int64_t *__restrict__ o1, int64_t total, const double *p0,
                       double *p1) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= total)
        return;
    const int64_t c = owner(o1, ncells, j);
    const int64_t blk = j - o1[c];
    const int64_t nb0 = o0[c + 1] - o0[c];
    double a[K + 1];
    for (int q = 0; q <= K; q++) a[q] = 0.0;
    const int64_t k1 = nb0 < (blk + 1) * kSumBlock ? nb0 : (blk + 1) * kSumBlock;
    for (int64_t k = blk * kSumBlock; k < k1; k++) {
        const double *s = p0 + (o0[c] + k) * (K + 1);
        for (int q = 0; q < K; q++) a[q] += s[q];
        a[K] = fmax(a[K], s[K]);
    }
    for (int q = 0; q <= K; q++) p1[j * (K + 1) + q] = a[q];
}

// Level 2 of pass 1: the centre of mass (nlnhost.cpp compute_moments).
__global__ void k_sum2_mass(const Cells C, int64_t ncells, const int64_t *__restrict__ o1,
                            const double *p1, double *cen, double *mass) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells)
        return;
    double a[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t k = o1[c]; k < o1[c + 1]; k++)
        for (int q = 0; q < 4; q++) a[q] += p1[k * 5 + q];
    const double m = a[0];
    for (int d = 0; d < 3; d++) cen[3 * c + d] = C.gc[3 * c + d] + (m > 0 ? a[1 + d] / m : 0.0);
    mass[c] = m;
}

// Level 2 of pass 2, then the cell's table records and critical radii and
// its walk record.
__global__ void k_sum2_tables(const Cells C, int64_t ncells, int64_t n,
                              const int64_t *__restrict__ o1, const double *p1, const double *cen,
                              const double *mass, nln_mac P, float4 *points, nln_qcell *qc,
                              nln_hcell *hc, nln_wcell *wc) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells)
        return;
    constexpr int K = NLN_NMOM;
    double mo[K];
    for (int q = 0; q < K; q++) mo[q] = 0.0;
    double bmax2 = 0.0;
    for (int64_t k = o1[c]; k < o1[c + 1]; k++) {
        for (int q = 0; q < K; q++) mo[q] += p1[k * (K + 1) + q];
        bmax2 = fmax(bmax2, p1[k * (K + 1) + K]);
    }
    const double cc[3] = {cen[3 * c], cen[3 * c + 1], cen[3 * c + 2]};
    const double m = mass[c], bmax = sqrt(bmax2);
    nln_qcell q;
    nln_hcell h;
    float pt[4];
    nln_cell_tables(cc, m, bmax, mo, pt, &q, &h);
    points[n + c] = make_float4(pt[0], pt[1], pt[2], pt[3]);
    qc[c] = q;
    hc[c] = h;
    double rc[3];
    nln_cell_rcrit(P, C.count[c], m, bmax, mo[31], mo[32], mo[33], rc);
    nln_wcell w;
    for (int d = 0; d < 3; d++) w.cen[d] = cc[d];
    w.bmax = bmax;
    for (int d = 0; d < 3; d++) w.rc[d] = rc[d];
    w.first = C.first[c];
    w.count = C.count[c];
    w.child = C.child[c];
    w.nchild = C.nchild[c];
    w.pad = 0;
    wc[c] = w;
}

// ------------------------------------------------------------ sink groups
// The runs of nlnhost.cpp collect_groups: the root alone when it is small
// (<= gmax bodies, or a leaf); for every large cell, its small children in
// order, adjacent ones merged while the run stays within gmax.
__global__ void k_runs(const Cells C, int64_t ncells, int gmax, int64_t *nruns, int64_t *rfirst,
                       int32_t *rcount) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells)
        return;
    const bool small = C.count[c] <= gmax || C.child[c] < 0;
    int nr = 0;
    if (small) {
        if (c == 0) {
            rfirst[0] = C.first[0];
            rcount[0] = C.count[0];
            nr = 1;
        }
    } else {
        int64_t mf = -1;
        int32_t mc = 0;
        for (int k = 0; k < C.nchild[c]; k++) {
            const int64_t d = C.child[c] + k;
            if (C.count[d] > gmax && C.child[d] >= 0)
                continue;
            if (mf >= 0 && mf + mc == C.first[d] && mc + C.count[d] <= gmax) {
                mc += C.count[d];
            } else {
                if (mf >= 0) {
                    rfirst[8 * c + nr] = mf;
                    rcount[8 * c + nr] = mc;
                    nr++;
                }
                mf = C.first[d];
                mc = C.count[d];
            }
        }
        if (mf >= 0) {
            rfirst[8 * c + nr] = mf;
            rcount[8 * c + nr] = mc;
            nr++;
        }
    }
    nruns[c] = nr;
}

__global__ void k_runs_compact(int64_t ncells, const int64_t *nruns, const int64_t *roff,
                               const int64_t *rfirst, const int32_t *rcount, int64_t *first,
                               int32_t *count) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells)
        return;
    for (int r = 0; r < nruns[c]; r++) {
        first[roff[c] + r] = rfirst[8 * c + r];
        count[roff[c] + r] = rcount[8 * c + r];
    }
}

// Runs longer than gmax (a leaf of coincident bodies that cannot split) as
// consecutive pieces of gmax bodies, the last one the remainder, as
// nlnhost.cpp splits them: pieces of run r start at poff[r].
__global__ void k_run_pieces(int64_t nr, const int64_t *rfirst, const int32_t *rcount,
                             const int64_t *poff, int gmax, int64_t *first, int32_t *count) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nr)
        return;
    int64_t o = poff[r];
    for (int32_t k = 0; k < rcount[r]; k += gmax) {
        first[o] = rfirst[r] + k;
        count[o] = rcount[r] - k < gmax ? rcount[r] - k : gmax;
        o++;
    }
}

__global__ void k_piece_count(int64_t nr, const int32_t *rcount, int gmax, int64_t *np) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nr)
        np[r] = (rcount[r] + gmax - 1) / gmax;
}

// Group records: FP64 centre of mass of its sinks in order, radius.
__global__ void k_groups(int64_t ng, const int64_t *first, const int32_t *count,
                         const float *spos, const float *smass, nln_group *groups) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ng)
        return;
    const int64_t f = first[g];
    const int32_t cnt = count[g];
    const float *P = spos + 3 * f;
    const float *M = smass + f;
    double m = 0, s[3] = {0, 0, 0};
    for (int32_t k = 0; k < cnt; k++) {
        m += M[k];
        for (int d = 0; d < 3; d++) s[d] += M[k] * (double)P[3 * k + d];
    }
    nln_group G;
    double r2max = 0;
    for (int d = 0; d < 3; d++) G.cen[d] = m > 0 ? s[d] / m : (double)P[d];
    for (int32_t k = 0; k < cnt; k++) {
        double r2 = 0;
        for (int d = 0; d < 3; d++) {
            const double x = (double)P[3 * k + d] - G.cen[d];
            r2 += x * x;
        }
        r2max = fmax(r2max, r2);
    }
    G.first = f;
    G.count = cnt;
    G.radius = (float)(sqrt(r2max) * (1.0 + 1e-6));
    groups[g] = G;
}

// ------------------------------------------------------------ walk
struct CountEmit {
    int64_t np = 0, nq = 0, nh = 0, nc = 0, nb = 0;
    __device__ void p(uint32_t, bool body) {
        np++;
        nb += body ? 1 : 0;
    }
    __device__ void q(uint32_t) { nq++; }
    __device__ void h(uint32_t) { nh++; }
    __device__ void c(uint32_t) { nc++; }
};

// Writes stay inside the group's counted ranges (ends E*): a walk that
// produced more entries than it counted only moves its cursor on, and the
// mismatch is reported.
struct FillEmit {
    uint32_t *P, *Q, *H, *Cl;
    uint32_t *EP, *EQ, *EH, *EC;
    __device__ void p(uint32_t e, bool) {
        if (P < EP)
            *P = e;
        P++;
    }
    __device__ void q(uint32_t e) {
        if (Q < EQ)
            *Q = e;
        Q++;
    }
    __device__ void h(uint32_t e) {
        if (H < EH)
            *H = e;
        H++;
    }
    __device__ void c(uint32_t e) {
        if (Cl < EC)
            *Cl = e;
        Cl++;
    }
};

// cnt: 5 per group (point, quadrupole, order-4, correction entries, bodies among the points)
__global__ void k_walk_count(const nln_wcell *__restrict__ wc, const float *spos, int64_t n,
                             const nln_group *__restrict__ groups, int64_t ng, nln_mac P,
                             int64_t *cnt, unsigned *err) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ng)
        return;
    int32_t stack[NLN_WALK_STACK];
    CountEmit em;
    const nln_group G = groups[g];
    if (nln_walk_group(wc, spos, n, G, P, stack, NLN_WALK_STACK, em))
        atomicOr(err, 1u);
    cnt[5 * g] = em.np;
    cnt[5 * g + 1] = em.nq;
    cnt[5 * g + 2] = em.nh;
    cnt[5 * g + 3] = em.nc;
    cnt[5 * g + 4] = em.nb;
}

__global__ void k_walk_fill(const nln_wcell *__restrict__ wc, const float *spos, int64_t n,
                            const nln_group *__restrict__ groups, int64_t ng, nln_mac P,
                            const int64_t *pp, const int64_t *qp, const int64_t *hp,
                            const int64_t *cp, uint32_t *pl, uint32_t *ql, uint32_t *hl,
                            uint32_t *cl, unsigned *err) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ng)
        return;
    int32_t stack[NLN_WALK_STACK];
    FillEmit em{pl + pp[g],     ql + qp[g],     hl + hp[g],     cl + cp[g],
                pl + pp[g + 1], ql + qp[g + 1], hl + hp[g + 1], cl + cp[g + 1]};
    const nln_group G = groups[g];
    if (nln_walk_group(wc, spos, n, G, P, stack, NLN_WALK_STACK, em))
        atomicOr(err, 1u);
    // the count pass sized every list: a walk that writes more or less is an error
    if (em.P != pl + pp[g + 1] || em.Q != ql + qp[g + 1] || em.H != hl + hp[g + 1] ||
        em.Cl != cl + cp[g + 1])
        atomicOr(err, 2u);
}

template <typename T>
int exclusive_scan(Bufs &B, const T *in, T *out, int64_t n, cudaStream_t st) {
    size_t bytes = 0;
    BC(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, (int)n, st));
    void *tmp = nullptr;
    BC(B.get((unsigned char **)&tmp, bytes));
    BC(cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, (int)n, st));
    B.drop(tmp);
    return 0;
}

}  // namespace

void dev_tree_free(DevTree &t, cudaMemPool_t pool) {
    void *ps[] = {t.points, t.qcells, t.hcells, t.groups, t.list[0], t.list[1], t.list[2],
                  t.list[3], t.order, t.cell_first, t.cell_count, t.cell_child, t.cell_nchild,
                  t.cell_level};
    for (void *p : ps)
        if (p) {
            if (pool)
                cudaFreeAsync(p, 0);
            else
                cudaFree(p);
        }
    t = DevTree{};
}

int gpu_tree_build(const nln_params &p, const float4 *bodies, int64_t n, cudaStream_t st,
                   DevTree &out, cudaMemPool_t pool) {
    out = DevTree{};
    if (!bodies || n <= 0)
        return gc::set_status(-1, "GPU tree build: no bodies");
    if (p.leaf_max < 1 || p.leaf_max > 65535 || p.group_max < 1 || p.group_max > 64 ||
        p.tol <= 0.0 || p.p2cut < 0 || p.p4cut < 0)
        return gc::set_status(-1, "GPU tree build: bad parameters (leaf_max 1..65535, group_max "
                                  "1..64, tol > 0)");
    if (n + 1 >= (int64_t)NLN_IDX_MASK || n >= (int64_t)INT32_MAX)
        return gc::set_status(-1, "GPU tree build: too many bodies for 27-bit list indices");
    Bufs B;
    B.pool = pool;
    B.st = st;
    out.pool = pool;
    double t0 = now_s();
    // ---- bounding cube (the host arithmetic of nln_tree_build)
    const unsigned bb = 592;
    float *blo = nullptr, *bhi = nullptr;
    unsigned *flag = nullptr;
    BC(B.get(&blo, 3 * bb));
    BC(B.get(&bhi, 3 * bb));
    BC(B.get(&flag, 4));
    BC(cudaMemsetAsync(flag, 0, 4 * sizeof(unsigned), st));
    k_bbox<<<bb, kThreads, 0, st>>>(bodies, n, p.box, blo, bhi, flag);
    BC(cudaGetLastError());
    std::vector<float> hlo(3 * bb), hhi(3 * bb);
    unsigned hbad = 0;
    BC(cudaMemcpyAsync(hlo.data(), blo, 3 * bb * sizeof(float), cudaMemcpyDeviceToHost, st));
    BC(cudaMemcpyAsync(hhi.data(), bhi, 3 * bb * sizeof(float), cudaMemcpyDeviceToHost, st));
    BC(cudaMemcpyAsync(&hbad, flag, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    BC(cudaStreamSynchronize(st));
    if (hbad)
        return gc::set_status(-1, p.box > 0 ? "GPU tree build: periodic body outside [0, box)"
                                            : "GPU tree build: non-finite position");
    double origin[3] = {0, 0, 0}, side = 0;
    if (p.box > 0) {
        side = p.box;
    } else {
        double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (unsigned k = 0; k < bb; k++)
            for (int d = 0; d < 3; d++) {
                lo[d] = std::min(lo[d], (double)hlo[3 * k + d]);
                hi[d] = std::max(hi[d], (double)hhi[3 * k + d]);
            }
        double ext = 0;
        for (int d = 0; d < 3; d++) ext = std::max(ext, hi[d] - lo[d]);
        ext = ext > 0 ? ext * (1.0 + 1e-5) : 1.0;
        for (int d = 0; d < 3; d++) origin[d] = 0.5 * (lo[d] + hi[d]) - 0.5 * ext;
        side = ext;
    }
    // ---- keys, stable sort by (key, index), bodies in tree order
    const double scale = (double)(1u << KEY_LEVELS) / side;
    uint64_t *k_in = nullptr, *k_out = nullptr;
    int64_t *i_in = nullptr;
    BC(B.get(&k_in, n));
    BC(B.get(&k_out, n));
    BC(B.get(&i_in, n));
    BC(B.get(&out.order, n));
    k_keys<<<grid_of(n), kThreads, 0, st>>>(bodies, n, origin[0], origin[1], origin[2], scale,
                                             k_in, i_in);
    BC(cudaGetLastError());
    {
        size_t bytes = 0;
        BC(cub::DeviceRadixSort::SortPairs(nullptr, bytes, k_in, k_out, i_in, out.order, (int)n, 0,
                                           64, st));
        unsigned char *tmp = nullptr;
        BC(B.get(&tmp, bytes));
        BC(cub::DeviceRadixSort::SortPairs(tmp, bytes, k_in, k_out, i_in, out.order, (int)n, 0, 64,
                                           st));
        B.drop(tmp);
    }
    B.drop(k_in);
    B.drop(i_in);
    float *spos = nullptr, *smass = nullptr;
    BC(B.get(&spos, 3 * n));
    BC(B.get(&smass, n));
    // the point table is sized once the cells are known: bodies go to a
    // temporary float4 array first
    float4 *bpts = nullptr;
    BC(B.get(&bpts, n));
    k_permute<<<grid_of(n), kThreads, 0, st>>>(bodies, out.order, n, spos, smass, bpts);
    BC(cudaGetLastError());
    BC(cudaStreamSynchronize(st));
    out.seconds[0] = now_s() - t0;
    t0 = now_s();

    // ---- cells, level by level
    int64_t cap = std::max<int64_t>(1024, 2 * (n / std::max(1, p.leaf_max)) + 64);
    Cells C{};
    auto alloc_cells = [&](Cells &D, int64_t c) -> int {
        BC(B.get(&D.first, c));
        BC(B.get(&D.count, c));
        BC(B.get(&D.child, c));
        BC(B.get(&D.nchild, c));
        BC(B.get(&D.level, c));
        BC(B.get(&D.gc, 3 * c));
        BC(B.get(&D.side, c));
        return 0;
    };
    if (int rc = alloc_cells(C, cap))
        return rc;
    {
        const int64_t f0 = 0;
        const int32_t cn = (int32_t)n, ch = -1, nch = 0, lv = 0;
        double g[3];
        for (int d = 0; d < 3; d++) g[d] = origin[d] + 0.5 * side;
        BC(cudaMemcpyAsync(C.first, &f0, sizeof(f0), cudaMemcpyHostToDevice, st));
        BC(cudaMemcpyAsync(C.count, &cn, sizeof(cn), cudaMemcpyHostToDevice, st));
        BC(cudaMemcpyAsync(C.child, &ch, sizeof(ch), cudaMemcpyHostToDevice, st));
        BC(cudaMemcpyAsync(C.nchild, &nch, sizeof(nch), cudaMemcpyHostToDevice, st));
        BC(cudaMemcpyAsync(C.level, &lv, sizeof(lv), cudaMemcpyHostToDevice, st));
        BC(cudaMemcpyAsync(C.gc, g, sizeof(g), cudaMemcpyHostToDevice, st));
        BC(cudaMemcpyAsync(C.side, &side, sizeof(side), cudaMemcpyHostToDevice, st));
        BC(cudaStreamSynchronize(st));
    }
    int64_t lo = 0, hi = 1;
    while (hi > lo) {
        const int64_t nf = hi - lo;
        int64_t *nk = nullptr, *bounds = nullptr, *off = nullptr;
        BC(B.get(&nk, nf));
        BC(B.get(&off, nf));
        BC(B.get(&bounds, 9 * nf));
        k_split_count<<<grid_of(nf), kThreads, 0, st>>>(C, lo, nf, k_out, p.leaf_max, nk, bounds);
        BC(cudaGetLastError());
        if (int rc = exclusive_scan(B, nk, off, nf, st))
            return rc;
        int64_t last_off = 0, last_nk = 0;
        BC(cudaMemcpyAsync(&last_off, off + nf - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        BC(cudaMemcpyAsync(&last_nk, nk + nf - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        BC(cudaStreamSynchronize(st));
        const int64_t total = last_off + last_nk;
        if (total > 0) {
            if (hi + total > cap) {  // grow the cell arrays
                int64_t ncap = std::max(2 * cap, hi + total + 1024);
                Cells D{};
                if (int rc = alloc_cells(D, ncap))
                    return rc;
                BC(cudaMemcpyAsync(D.first, C.first, hi * sizeof(int64_t), cudaMemcpyDeviceToDevice, st));
                BC(cudaMemcpyAsync(D.count, C.count, hi * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
                BC(cudaMemcpyAsync(D.child, C.child, hi * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
                BC(cudaMemcpyAsync(D.nchild, C.nchild, hi * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
                BC(cudaMemcpyAsync(D.level, C.level, hi * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
                BC(cudaMemcpyAsync(D.gc, C.gc, 3 * hi * sizeof(double), cudaMemcpyDeviceToDevice, st));
                BC(cudaMemcpyAsync(D.side, C.side, hi * sizeof(double), cudaMemcpyDeviceToDevice, st));
                BC(cudaStreamSynchronize(st));
                B.drop(C.first); B.drop(C.count); B.drop(C.child); B.drop(C.nchild);
                B.drop(C.level); B.drop(C.gc); B.drop(C.side);
                C = D;
                cap = ncap;
            }
            k_split_write<<<grid_of(nf), kThreads, 0, st>>>(C, lo, nf, nk, bounds, off, hi);
            BC(cudaGetLastError());
        }
        B.drop(nk);
        B.drop(off);
        B.drop(bounds);
        lo = hi;
        hi += total;
    }
    const int64_t nc = hi;
    if (n + nc + 1 >= (int64_t)NLN_IDX_MASK)
        return gc::set_status(-1, "GPU tree build: bodies plus cells exceed 27-bit list indices");
    out.n = n;
    out.ncells = nc;
    out.box = p.box;
    BC(cudaStreamSynchronize(st));
    out.seconds[1] = now_s() - t0;
    t0 = now_s();

    // ---- moments: block offsets of the canonical sums
    int64_t *o0 = nullptr, *o1 = nullptr, *nb = nullptr;
    BC(B.get(&o0, nc + 1));
    BC(B.get(&o1, nc + 1));
    BC(B.get(&nb, nc + 1));
    std::vector<int32_t> hcount(nc);
    BC(cudaMemcpyAsync(hcount.data(), C.count, nc * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    BC(cudaStreamSynchronize(st));
    std::vector<int64_t> ho0(nc + 1), ho1(nc + 1);
    ho0[0] = ho1[0] = 0;
    for (int64_t c = 0; c < nc; c++) {
        const int64_t b0 = (hcount[c] + kSumBlock - 1) / kSumBlock;
        ho0[c + 1] = ho0[c] + b0;
        ho1[c + 1] = ho1[c] + (b0 + kSumBlock - 1) / kSumBlock;
    }
    BC(cudaMemcpyAsync(o0, ho0.data(), (nc + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    BC(cudaMemcpyAsync(o1, ho1.data(), (nc + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    const int64_t B0 = ho0[nc], B1 = ho1[nc];
    double *cen = nullptr, *mass = nullptr, *p0 = nullptr, *p1 = nullptr;
    BC(B.get(&cen, 3 * nc));
    BC(B.get(&mass, nc));
    // pass 1: centre of mass
    BC(B.get(&p0, B0 * 5));
    BC(B.get(&p1, B1 * 5));
    k_sum0<4><<<grid_of(B0), kThreads, 0, st>>>(C, nc, o0, B0, spos, smass, C.gc, p0);
    BC(cudaGetLastError());
    k_sum1<4><<<grid_of(B1), kThreads, 0, st>>>(C, nc, o0, o1, B1, p0, p1);
    BC(cudaGetLastError());
    k_sum2_mass<<<grid_of(nc), kThreads, 0, st>>>(C, nc, o1, p1, cen, mass);
    BC(cudaGetLastError());
    BC(cudaStreamSynchronize(st));
    B.drop(p0);
    B.drop(p1);
    // pass 2: raw moments, tables, critical radii, walk records
    constexpr int K2 = NLN_NMOM + 1;
    BC(B.get(&p0, B0 * K2));
    BC(B.get(&p1, B1 * K2));
    k_sum0<NLN_NMOM><<<grid_of(B0), kThreads, 0, st>>>(C, nc, o0, B0, spos, smass, cen, p0);
    BC(cudaGetLastError());
    k_sum1<NLN_NMOM><<<grid_of(B1), kThreads, 0, st>>>(C, nc, o0, o1, B1, p0, p1);
    BC(cudaGetLastError());
    BC(B.get(&out.points, n + nc));
    BC(B.get(&out.qcells, nc));
    BC(B.get(&out.hcells, nc));
    nln_wcell *wc = nullptr;
    BC(B.get(&wc, nc));
    BC(cudaMemcpyAsync(out.points, bpts, n * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    nln_mac P;
    P.tol = p.tol;
    P.rel_tol = p.rel_tol;
    P.rel_tol0 = p.rel_tol0;
    P.ptol_boost = p.ptol_boost;
    P.bmax0 = 0.5 * side;
    P.p2cut = p.p2cut;
    P.p4cut = p.p4cut;
    P.box = p.box;
    P.ewald_theta = p.ewald_theta;
    k_sum2_tables<<<grid_of(nc), kThreads, 0, st>>>(C, nc, n, o1, p1, cen, mass, P, out.points,
                                                     out.qcells, out.hcells, wc);
    BC(cudaGetLastError());
    BC(cudaStreamSynchronize(st));
    B.drop(p0);
    B.drop(p1);
    B.drop(bpts);
    B.drop(cen);
    B.drop(mass);
    B.drop(o0);
    B.drop(o1);
    B.drop(nb);
    out.seconds[2] = now_s() - t0;
    t0 = now_s();

    // ---- sink groups
    int32_t *rcount = nullptr, *gcount = nullptr;
    int64_t *nruns = nullptr, *rfirst = nullptr, *roff = nullptr, *gfirst = nullptr;
    BC(B.get(&nruns, nc + 1));
    BC(B.get(&rcount, 8 * nc));
    BC(B.get(&rfirst, 8 * nc));
    BC(B.get(&roff, nc + 1));
    BC(cudaMemsetAsync(nruns, 0, (nc + 1) * sizeof(int64_t), st));
    k_runs<<<grid_of(nc), kThreads, 0, st>>>(C, nc, p.group_max, nruns, rfirst, rcount);
    BC(cudaGetLastError());
    if (int rc = exclusive_scan(B, nruns, roff, nc + 1, st))  // roff[nc] = the run count
        return rc;
    int64_t ng = 0;
    BC(cudaMemcpyAsync(&ng, roff + nc, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    BC(cudaStreamSynchronize(st));
    if (ng <= 0)
        return gc::set_status(-1, "GPU tree build: no sink groups");
    int64_t *ufirst = nullptr;
    int32_t *ucount = nullptr;
    BC(B.get(&ufirst, ng));
    BC(B.get(&ucount, ng));
    BC(B.get(&gfirst, ng));
    BC(B.get(&gcount, ng));
    k_runs_compact<<<grid_of(nc), kThreads, 0, st>>>(nc, nruns, roff, rfirst, rcount, ufirst,
                                                      ucount);
    BC(cudaGetLastError());
    {
        size_t bytes = 0;
        BC(cub::DeviceRadixSort::SortPairs(nullptr, bytes, ufirst, gfirst, ucount, gcount, (int)ng,
                                           0, 64, st));
        unsigned char *tmp = nullptr;
        BC(B.get(&tmp, bytes));
        BC(cub::DeviceRadixSort::SortPairs(tmp, bytes, ufirst, gfirst, ucount, gcount, (int)ng, 0,
                                           64, st));
        B.drop(tmp);
    }
    // split runs longer than group_max
    {
        int64_t *np = nullptr, *poff = nullptr;
        BC(B.get(&np, ng + 1));
        BC(B.get(&poff, ng + 1));
        BC(cudaMemsetAsync(np, 0, (ng + 1) * sizeof(int64_t), st));
        k_piece_count<<<grid_of(ng), kThreads, 0, st>>>(ng, gcount, p.group_max, np);
        BC(cudaGetLastError());
        if (int rc = exclusive_scan(B, np, poff, ng + 1, st))
            return rc;
        int64_t npieces = 0;
        BC(cudaMemcpyAsync(&npieces, poff + ng, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        BC(cudaStreamSynchronize(st));
        if (npieces != ng) {
            int64_t *pf = nullptr;
            int32_t *pc = nullptr;
            BC(B.get(&pf, npieces));
            BC(B.get(&pc, npieces));
            k_run_pieces<<<grid_of(ng), kThreads, 0, st>>>(ng, gfirst, gcount, poff, p.group_max,
                                                            pf, pc);
            BC(cudaGetLastError());
            gfirst = pf;
            gcount = pc;
            ng = npieces;
        }
    }
    BC(B.get(&out.groups, ng));
    k_groups<<<grid_of(ng), kThreads, 0, st>>>(ng, gfirst, gcount, spos, smass, out.groups);
    BC(cudaGetLastError());
    out.ngroups = ng;
    BC(cudaStreamSynchronize(st));
    out.seconds[3] = now_s() - t0;
    t0 = now_s();

    // ---- walk: count, offsets, fill
    int64_t *cnt = nullptr;
    BC(B.get(&cnt, 5 * ng));
    BC(cudaMemsetAsync(cnt, 0, 5 * ng * sizeof(int64_t), st));
    BC(cudaMemsetAsync(flag, 0, sizeof(unsigned), st));
    k_walk_count<<<grid_of(ng, 128), 128, 0, st>>>(wc, spos, n, out.groups, ng, P, cnt, flag);
    BC(cudaGetLastError());
    std::vector<int64_t> hc(5 * ng);
    BC(cudaMemcpyAsync(hc.data(), cnt, 5 * ng * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    BC(cudaMemcpyAsync(&hbad, flag, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    out.groups_h.resize(ng);
    BC(cudaMemcpyAsync(out.groups_h.data(), out.groups, ng * sizeof(nln_group),
                       cudaMemcpyDeviceToHost, st));
    BC(cudaStreamSynchronize(st));
    if (hbad)
        return gc::set_status(-1, "GPU tree build: a group's walk did not cover every body "
                                  "exactly once, or overflowed its stack");
    const double t_count = now_s() - t0;
    t0 = now_s();
    for (int k = 0; k < 4; k++) out.ptr_h[k].assign(ng + 1, 0);
    for (int64_t g = 0; g < ng; g++) {
        // a group's lists cover every body once: no kind can exceed the point table
        for (int k = 0; k < 5; k++)
            if (hc[5 * g + k] < 0 || hc[5 * g + k] > n + nc)
                return gc::set_status(-1, "GPU tree build: group %lld counted %lld entries",
                                      (long long)g, (long long)hc[5 * g + k]);
        for (int k = 0; k < 4; k++) out.ptr_h[k][g + 1] = out.ptr_h[k][g] + hc[5 * g + k];
        const int64_t c = out.groups_h[g].count, nbod = hc[5 * g + 4];
        out.counts[0] += c * nbod;
        out.counts[1] += c * (hc[5 * g] - nbod);
        out.counts[2] += c * hc[5 * g + 1];
        out.counts[3] += c * hc[5 * g + 2];
    }
    int64_t *dptr[4];
    for (int k = 0; k < 4; k++) {
        out.len[k] = out.ptr_h[k][ng];
        BC(B.get(&out.list[k], out.len[k]));
        BC(B.get(&dptr[k], ng + 1));
        BC(cudaMemcpyAsync(dptr[k], out.ptr_h[k].data(), (ng + 1) * sizeof(int64_t),
                           cudaMemcpyHostToDevice, st));
    }
    out.seconds[5] = now_s() - t0;  // offsets and list allocation
    t0 = now_s();
    BC(cudaMemsetAsync(flag, 0, sizeof(unsigned), st));
    k_walk_fill<<<grid_of(ng, 128), 128, 0, st>>>(wc, spos, n, out.groups, ng, P, dptr[0], dptr[1],
                                              dptr[2], dptr[3], out.list[0], out.list[1],
                                              out.list[2], out.list[3], flag);
    BC(cudaGetLastError());
    BC(cudaMemcpyAsync(&hbad, flag, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    BC(cudaStreamSynchronize(st));
    if (hbad)
        return gc::set_status(-1, "GPU tree build: the filling walk differs from the counting "
                                  "walk (0x%x)", hbad);
    out.seconds[4] = t_count + (now_s() - t0);
    // ---- the tree links, handed on
    out.cell_first = C.first;
    out.cell_count = C.count;
    out.cell_child = C.child;
    out.cell_nchild = C.nchild;
    out.cell_level = C.level;
    void *keep[] = {out.points, out.qcells, out.hcells, out.groups, out.list[0], out.list[1],
                    out.list[2], out.list[3], out.order, C.first, C.count, C.child, C.nchild,
                    C.level};
    for (void *q : keep) B.release(q);
    return 0;
}
