// batch.cu -- Part 2 of gravcuda.h: every sink group of a step evaluated
// by persistent kernels from length-sorted work queues, on index lists into
// device-resident point and cell tables.
//
// Mixed precision (none of this exists in the reference, whose lists carry
// absolute FP32 copies, nln/mac.c:1421-1561):
//   * each sink is held as an FP32 offset from its group's FP64 centre;
//   * each source record is re-centred on the same FP64 centre (with its
//     periodic image shift) as it is staged, so the inner loops subtract
//     two small FP32 numbers;
//   * partial sums of one staged tile are plain FP32, folded into a
//     compensated (hi, lo) accumulator per tile;
//   * work-item partials are combined per group in FP64, in a fixed order.
// Work decomposition: a work item is (group, kind, range of its list);
// long lists are split so that small problems still fill the GPU; every
// warp pulls items (costliest first) from its kind's queue until it is
// empty.  One warp owns one item: lane = sink, 32 sources per staged tile;
// tiles are staged by TMA row gathers (cp.async.bulk.tensor tile::gather4
// over a 2-D tensor map of the table, one instruction per 4 records, issued
// by one lane) into a 2-4 stage ring signalled by per-warp mbarriers.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <mutex>
#include <numeric>
#include <vector>

#include "build.cuh"
#include "common.cuh"
#include "gravcuda.h"
#include "ewald.cuh"
#define NLN_EWALD_NO_EXPORT
#include "host/ewald_table.cpp"
#include "interact.cuh"

namespace {

enum { KP = 0, KQ = 1, KH = 2 };
constexpr int TILE = 32;

struct Item {
    int32_t group;
    int32_t slot;      // partial-result slot (creation order: grouped by group)
    int64_t begin, end;
};

// One group's correction moments as k_ewald_moments stores them (EwMoments).
struct EwStored {
    double lo[10];
    float hi[25];
    float pad[3];
};

struct DevProblem {
    const float4 *points;
    const nln_qcell *qcells;
    const nln_hcell *hcells;
    const nln_group *groups;
    const uint32_t *list[3];   // idx | shift << 27
    int64_t ntab[3];           // table sizes for bounds checks
    const Item *items[3];
    int nitems[3];
    int *counters;             // 3 queue heads
    float4 *part;              // nslots x 32 lanes x 2 (hi, lo)
    const int64_t *gslot;      // ngroups + 1: slots of group g
    float4 *out;               // nbodies
    int64_t ngroups;           // k_finish covers groups gbegin .. ngroups-1
    int64_t gbegin;
    int64_t ncells;
    float eps2;
    float qsh;
    double box;
    unsigned *err;
    // periodic correction
    const int64_t *cptr;       // per-group offsets of the correction list
    const uint32_t *clist;     // correction list: point-table record | image << 27
    int ewald;
    EwTab ew;
    float ew_self;             // C(0) - pi/(alpha^2 L^3): the self term ewald() leaves out
    float ew_trace;            // trace of the Hessian of C: -4 pi / L^3
    EwStored *ewm;             // per-group moments from k_ewald_moments
    // FP64 centres of the cells for the point table's monopole records (the
    // mixed form re-centres them like every other source): a pre-staged cell
    // table (centre x, y in floats 0-3, z in floats 10-11 of each record of
    // cstride float4s), or null, where the FP32 point record is used
    const float4 *cstage;
    int cstride;
};

template <int KIND, bool PAIRED = false>
struct KindOf {
    static constexpr int rec_bytes = KIND == KP ? 16 : (KIND == KQ ? 64 : 128);
    static constexpr int order = KIND == KP ? 0 : (KIND == KQ ? 2 : 4);
    // pipeline depth: short per-record work needs more copies in flight; the
    // paired order-4 path frees its one stage as soon as the tile is
    // re-laid into the pair buffer, so the next copy overlaps the compute
    static constexpr int stages = PAIRED ? 1 : (KIND == KP ? 4 : (KIND == KQ ? 3 : 2));
    // one TMA row gather brings 4 records; each lands 128-byte aligned
    static constexpr int group_bytes = 4 * rec_bytes < 128 ? 128 : 4 * rec_bytes;
    static constexpr int stage_bytes = (TILE / 4) * group_bytes;
    // paired tiles: 16 record pairs of 32 (order 4) or 10 (quadrupole)
    // interleaved fields, one pair every 68 or 20 floats (16-byte aligned;
    // the re-lay's 8-byte stores of a half-warp hit distinct banks)
    static constexpr int pair_fields = KIND == KH ? 32 : 10;
    static constexpr int pair_stride = pair_fields == 32 ? 68 : 20;
    static constexpr int pair_bytes = PAIRED ? (TILE / 2) * pair_stride * 4 : 0;
    // per-warp shared memory: stages of 32 records, the pair buffer,
    // mbarriers, image codes
    static constexpr int warp_bytes =
        (stages * stage_bytes + pair_bytes + stages * 8 + stages * TILE * 4 + 127) / 128 * 128;
    // byte offset of record r inside a stage
    static __device__ __forceinline__ int rec_off(int r) {
        return (r >> 2) * group_bytes + (r & 3) * rec_bytes;
    }
};

__device__ __forceinline__ void decode_shift(uint32_t code, double box, double &sx, double &sy,
                                             double &sz) {
    sx = ((int)(code / 9) - 1) * box;
    sy = ((int)(code / 3 % 3) - 1) * box;
    sz = ((int)(code % 3) - 1) * box;
}

// Convert this lane's record (just landed by TMA) in place into the staged
// form of interact.cuh, re-centred on the group centre c.  STAGED: the cell
// tables are pre-staged (k_stage_cells) and only the 16-byte header (FP64
// centre -> FP32 offset, mass) is rewritten; otherwise the raw nln_qcell /
// nln_hcell record is scaled here.
template <int KIND, bool STAGED>
__device__ __forceinline__ void convert(unsigned char *slot, uint32_t code, const double *c,
                                        double box) {
    double sx, sy, sz;
    decode_shift(code, box, sx, sy, sz);
    float *o = reinterpret_cast<float *>(slot);
    if (KIND == KP) {
        float4 p = *reinterpret_cast<const float4 *>(slot);
        o[0] = (float)((double)p.x + sx - c[0]);
        o[1] = (float)((double)p.y + sy - c[1]);
        o[2] = (float)((double)p.z + sz - c[2]);
        o[3] = p.w;
    } else if (STAGED) {
        const double *d = reinterpret_cast<const double *>(slot);
        const double cx = d[0], cy = d[1], cz = d[5];
        const float m = o[KIND == KQ ? 12 : 31];
        *reinterpret_cast<float4 *>(slot) =
            make_float4((float)(cx + sx - c[0]), (float)(cy + sy - c[1]), (float)(cz + sz - c[2]), m);
    } else if (KIND == KQ) {
        const nln_qcell q = *reinterpret_cast<const nln_qcell *>(slot);
        o[0] = (float)(q.cen[0] + sx - c[0]);
        o[1] = (float)(q.cen[1] + sy - c[1]);
        o[2] = (float)(q.cen[2] + sz - c[2]);
        o[3] = q.mass;
        float q2[5] = {q.qxx, q.qxy, q.qyy, q.qxz, q.qyz};
        stage_quad(o, q.R, q2);
    } else {
        const nln_hcell h = *reinterpret_cast<const nln_hcell *>(slot);
        o[0] = (float)(h.cen[0] + sx - c[0]);
        o[1] = (float)(h.cen[1] + sy - c[1]);
        o[2] = (float)(h.cen[2] + sz - c[2]);
        o[3] = h.mass;
        stage_quad(o, h.R, h.q2);
        stage_hexa(o, h.R, h.q3, h.q4);
    }
}

// Unpack the run-packed lists (format in nlnlists.h) of groups g0..g1-1,
// one warp per group.  Per 32-word block: a warp scan of the words' entry
// counts places each word's entries (an entry word stands for itself, a run
// word for the n entries after the word before it); then the warp writes
// the block's entries 32 consecutive ones at a time, each lane finding the
// word its entry comes from by a binary search over the scan.  Stores stay
// inside the group's plain range [ptr[g], ptr[g+1]); a group that does not
// fill it exactly, a run word that starts a group or follows a run word, or
// a run that would carry into the image code sets GC_DEV_BAD_RUNS.
__global__ void k_unpack(const uint32_t *__restrict__ z, const int64_t *__restrict__ zptr,
                         const int64_t *__restrict__ ptr, int64_t g0, int64_t g1,
                         uint32_t *__restrict__ out, unsigned *err) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t g = g0 + (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); g < g1;
         g += nwarps) {
        const int64_t zb = zptr[g], ze = zptr[g + 1], oe = ptr[g + 1];
        int64_t pos = ptr[g];
        uint32_t prev = 0;  // last word of the previous block
        bool have_prev = false, bad = false;
        for (int64_t b = zb; b < ze; b += 32) {
            const bool valid = b + lane < ze;
            const uint32_t w = valid ? z[b + lane] : 0u;
            const bool run = valid && (w >> NLN_IDX_BITS) == NLN_RUN_CODE;
            uint32_t before = __shfl_up_sync(FULL, w, 1);
            bool before_ok = true;
            if (lane == 0) {
                before = prev;
                before_ok = have_prev;
            }
            uint32_t cnt = !valid ? 0u : (run ? (w & NLN_IDX_MASK) : 1u);
            if (run && (!before_ok || (before >> NLN_IDX_BITS) == NLN_RUN_CODE || cnt == 0 ||
                        (before & NLN_IDX_MASK) + cnt > NLN_IDX_MASK)) {
                bad = true;
                cnt = 0;
            }
            const uint32_t first = run ? before + 1u : w;  // entry j of this word: first + j
            // block totals stay below 2^32: at most 32 words of 2^27 - 1
            uint32_t inc = cnt;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t v = __shfl_up_sync(FULL, inc, o);
                if (lane >= o)
                    inc += v;
            }
            const uint32_t total = __shfl_sync(FULL, inc, 31);
            if (pos + (int64_t)total > oe)
                bad = true;
            const int64_t room = oe - pos;
            const uint32_t lim = room <= 0 ? 0u : (room < (int64_t)total ? (uint32_t)room : total);
            for (uint32_t j0 = 0; j0 < lim; j0 += 32) {
                const uint32_t j = j0 + lane;
                // owner = number of words whose entries all lie before j
                int owner = 0;
#pragma unroll
                for (int step = 16; step >= 1; step >>= 1) {
                    const uint32_t v = __shfl_sync(FULL, inc, owner + step - 1);
                    if (v <= j)
                        owner += step;
                }
                owner = min(owner, 31);
                const uint32_t f = __shfl_sync(FULL, first, owner);
                const uint32_t s0 = __shfl_sync(FULL, inc - cnt, owner);
                if (j < lim)
                    out[pos + j] = f + (j - s0);
            }
            pos += total;
            prev = __shfl_sync(FULL, w, 31);
            have_prev = true;
        }
        if (pos != oe)
            bad = true;
        if (__any_sync(FULL, bad) && lane == 0)
            atomicOr(err, GC_DEV_BAD_RUNS);
    }
}

// Device-side check of an uploaded list, one warp per work item (or per
// group for the correction list): every entry's index inside its table and
// its image code in 0..26.  For the point list it also counts body and cell
// entries, weighted by the group's sinks.  acc: [0] error flag, [1] body
// interactions, [2] monopole-cell interactions.
__global__ void k_check_lists(const uint32_t *__restrict__ list, const Item *__restrict__ items,
                              int nitems, const int64_t *__restrict__ gptr, int64_t ngroups,
                              const nln_group *__restrict__ groups, uint32_t ntab, uint32_t nb,
                              int count_bodies, unsigned long long *acc) {
    const int lane = threadIdx.x & 31;
    const int64_t nwork = items ? nitems : ngroups;
    for (int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < nwork;
         w += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        int64_t b, e;
        int32_t g;
        if (items) {
            const Item it = items[w];
            b = it.begin;
            e = it.end;
            g = it.group;
        } else {
            b = gptr[w];
            e = gptr[w + 1];
            g = (int32_t)w;
        }
        unsigned bad = 0;
        long long nbody = 0;
        for (int64_t k = b + lane; k < e; k += 32) {
            const uint32_t v = list[k];
            const uint32_t idx = v & NLN_IDX_MASK;
            bad |= (idx >= ntab || (v >> NLN_IDX_BITS) > 26u) ? 1u : 0u;
            nbody += idx < nb ? 1 : 0;
        }
        bad = __reduce_or_sync(0xffffffffu, bad);
        for (int d = 16; d > 0; d >>= 1) nbody += __shfl_xor_sync(0xffffffffu, nbody, d);
        if (lane == 0) {
            if (bad)
                atomicOr(&acc[0], 1ull);
            if (count_bodies) {
                const long long c = groups[g].count;
                atomicAdd(&acc[1], (unsigned long long)(nbody * c));
                atomicAdd(&acc[2], (unsigned long long)((e - b - nbody) * c));
            }
        }
    }
}

// Pre-staged cell tables: the staged moments of interact.cuh at their
// offsets, with the FP64 centre and the mass in the slots the inner loops
// never read (centre x, y in floats 0-3 and z in floats 10-11; mass in
// float 12 (quadrupole, 16 floats) or 31 (order 4, 32 floats)), so that a
// tile's convert only rewrites the header.
__global__ void k_stage_cells(const nln_qcell *__restrict__ qc, const nln_hcell *__restrict__ hc,
                              int64_t n, float4 *__restrict__ qs, float4 *__restrict__ hs) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n)
        return;
    if (qs) {
        const nln_qcell q = qc[c];
        float o[16];
#pragma unroll
        for (int k = 0; k < 16; k++) o[k] = 0.f;
        const float q2[5] = {q.qxx, q.qxy, q.qyy, q.qxz, q.qyz};
        stage_quad(o, q.R, q2);
        memcpy(&o[0], &q.cen[0], 8);
        memcpy(&o[2], &q.cen[1], 8);
        memcpy(&o[10], &q.cen[2], 8);
        o[12] = q.mass;
#pragma unroll
        for (int k = 0; k < 4; k++) qs[c * 4 + k] = make_float4(o[4 * k], o[4 * k + 1], o[4 * k + 2], o[4 * k + 3]);
    }
    if (hs) {
        const nln_hcell h = hc[c];
        float o[32];
#pragma unroll
        for (int k = 0; k < 32; k++) o[k] = 0.f;
        stage_quad(o, h.R, h.q2);
        stage_hexa(o, h.R, h.q3, h.q4);
        memcpy(&o[0], &h.cen[0], 8);
        memcpy(&o[2], &h.cen[1], 8);
        memcpy(&o[10], &h.cen[2], 8);
        o[31] = h.mass;
#pragma unroll
        for (int k = 0; k < 8; k++) hs[c * 8 + k] = make_float4(o[4 * k], o[4 * k + 1], o[4 * k + 2], o[4 * k + 3]);
    }
}

// Re-lay this lane's pre-staged record (just landed by TMA at its stage
// slot) into the pair-interleaved tile of quad2_plummer / hexa2_plummer:
// header re-centred on the group centre c in the record's image; for order
// 4 the octupole and four hexadecapole fields negated as that layout wants.
// A lane past the tile's end writes a massless, momentless record far away,
// which adds exactly zero.  Lanes 2p and 2p+1 write pair p: one shuffle per
// field pair.
template <int KIND>
__device__ __forceinline__ void relay_pairs(const unsigned char *stage, uint32_t code, bool valid,
                                            const double *c, double box, float *pbuf, int lane) {
    using K = KindOf<KIND, true>;
    constexpr int NF = K::pair_fields;
    constexpr int NR = K::rec_bytes / 4;  // staged record floats
    float g[NF];
    if (valid) {
        const float4 *src = reinterpret_cast<const float4 *>(stage + K::rec_off(lane));
        float f[NR];
#pragma unroll
        for (int k = 0; k < NR / 4; k++) {
            const float4 v = src[k];
            f[4 * k] = v.x;
            f[4 * k + 1] = v.y;
            f[4 * k + 2] = v.z;
            f[4 * k + 3] = v.w;
        }
        double sx, sy, sz;
        decode_shift(code, box, sx, sy, sz);
        const double cx = __hiloint2double(__float_as_int(f[1]), __float_as_int(f[0]));
        const double cy = __hiloint2double(__float_as_int(f[3]), __float_as_int(f[2]));
        const double cz = __hiloint2double(__float_as_int(f[11]), __float_as_int(f[10]));
        g[0] = (float)(cx + sx - c[0]);
        g[1] = (float)(cy + sy - c[1]);
        g[2] = (float)(cz + sz - c[2]);
        g[3] = f[KIND == KH ? 31 : 12];
#pragma unroll
        for (int k = 4; k < 10; k++) g[k] = f[k];
        if (KIND == KH) {
            // h_z's xxz and yyz coefficients with -Xxxyy folded in (its
            // z z-trace terms): -(Xxxxx + Xxxyy), -(Xyyyy + Xxxyy)
            g[10] = -(f[21] + f[23]);
            g[11] = -(f[25] + f[23]);
#pragma unroll
            for (int k = 12; k < 19; k++) g[k] = -f[k];
            g[19] = f[19];
            g[20] = f[20];
#pragma unroll
            for (int k = 21; k < 30; k++) g[k] = f[k];
            g[30] = -f[30];
            g[31] = 0.f;
        }
    } else {
#pragma unroll
        for (int k = 0; k < NF; k++) g[k] = k < 3 ? 1.0e3f : 0.f;
    }
    const int s = lane & 1;
    float *dst = pbuf + (lane >> 1) * K::pair_stride + 2 * s;
#pragma unroll
    for (int q = 0; q < NF / 2; q++) {
        const float send = s ? g[2 * q] : g[2 * q + 1];
        const float recv = __shfl_xor_sync(0xffffffffu, send, 1);
        *reinterpret_cast<float2 *>(dst + 4 * q) =
            s ? make_float2(recv, g[2 * q + 1]) : make_float2(g[2 * q], recv);
    }
}

// Compile-time shape of the paired kernels, as measured best on a B200
// (-D to rebuild with others): unroll of the pair loop and minimum resident
// blocks (register cap) for the order-4 (H2) and quadrupole (Q2) kernels;
// GRAV_Q2_PAIRED=0 keeps the quadrupole kernel on the scalar loop.  Order 4:
// unroll 2 held to 3 blocks (80 registers, a few spilled words) is 0.6 %
// faster than unroll 1 and beat unroll 2 at its own 117 registers; minimum
// blocks 0 leaves the register count to the compiler (a 1 there lets it
// grow and cost occupancy).
#ifndef GRAV_H2_UNROLL
#define GRAV_H2_UNROLL 2
#endif
#ifndef GRAV_H2_MINB
#define GRAV_H2_MINB 3
#endif
#ifndef GRAV_Q2_MINB
#define GRAV_Q2_MINB 0
#endif
#ifndef GRAV_Q2_UNROLL
#define GRAV_Q2_UNROLL 4
#endif
#ifndef GRAV_Q2_PAIRED
#define GRAV_Q2_PAIRED 1
#endif
constexpr int kH2Unroll = GRAV_H2_UNROLL;
constexpr int kQ2Unroll = GRAV_Q2_UNROLL;
// PLAIN: the plain FP32 form the reference's lists compute in (absolute FP32
// coordinates, nln/mac.c:1421-1561 copies cell centres as floats): sinks and
// sources are not re-centred on the group centre and tile sums are added
// without compensation.  It exists to be compared with the mixed form.
template <int KIND, bool STAGED, bool PLAIN = false>
__global__ void __launch_bounds__(256, KIND == KH ? (STAGED ? GRAV_H2_MINB : 3)
                                                  : (KIND == KQ && STAGED ? GRAV_Q2_MINB : 0))
    k_batch(const __grid_constant__ CUtensorMap tmap, DevProblem P) {
    // staged quadrupole and order-4 tables run the paired (f32x2)
    // interaction on a pair-interleaved copy of each tile
    constexpr bool PAIRED = (KIND == KH || (KIND == KQ && GRAV_Q2_PAIRED)) && STAGED;
    using K = KindOf<KIND, PAIRED>;
    constexpr int RB = K::rec_bytes;
    constexpr int ORDER = K::order;
    constexpr int NST = K::stages;
    extern __shared__ __align__(128) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    unsigned char *wbuf = smem + (size_t)wib * K::warp_bytes;
    float *pbuf = reinterpret_cast<float *>(wbuf + NST * K::stage_bytes);  // paired path
    uint64_t *bar = reinterpret_cast<uint64_t *>(wbuf + NST * K::stage_bytes + K::pair_bytes);
    uint32_t *codes = reinterpret_cast<uint32_t *>(bar + NST);  // [NST][TILE] image codes
    if (lane == 0) {
        for (int s = 0; s < NST; s++) mbar_init(&bar[s], 1);
        fence_mbar_init();
    }
    __syncwarp();

    const uint32_t *list = P.list[KIND];
    const uint32_t ntab = (uint32_t)P.ntab[KIND];
    // tiles issued (and later consumed, in the same order) by this warp:
    // tile seq uses stage seq % NST with mbarrier parity (seq / NST) & 1
    uint32_t tseq = 0;
    bool alive = true;

    while (alive) {
        int it = 0;
        if (lane == 0)
            it = atomicAdd(&P.counters[KIND], 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= P.nitems[KIND])
            break;
        const Item item = P.items[KIND][it];
        const nln_group G = P.groups[item.group];
        const double c[3] = {PLAIN ? 0.0 : G.cen[0], PLAIN ? 0.0 : G.cen[1],
                             PLAIN ? 0.0 : G.cen[2]};
        // this lane's sink, as an FP32 offset from the group centre
        float ux = 0.f, uy = 0.f, uz = 0.f;
        if (lane < G.count) {
            float4 s = P.points[G.first + lane];
            ux = (float)((double)s.x - c[0]);
            uy = (float)((double)s.y - c[1]);
            uz = (float)((double)s.z - c[2]);
        }
        float hi[4] = {0.f, 0.f, 0.f, 0.f}, lo[4] = {0.f, 0.f, 0.f, 0.f};
        const int64_t nent = item.end - item.begin;
        const int ntile = (int)((nent + TILE - 1) / TILE);

        auto fetch = [&](int t) -> uint32_t {
            int64_t k = item.begin + (int64_t)t * TILE + lane;
            return (t < ntile && k < item.end) ? __ldg(list + k) : 0u;
        };
        // Start tile t (sequence number seq): each lane holds one entry; the
        // row indices are gathered to lane 0, which issues one TMA row
        // gather per 4 records.  Unused rows of a short tile repeat row 0.
        auto issue = [&](int t, uint32_t ent, uint32_t seq) {
            const int nt = (int)min((int64_t)TILE, nent - (int64_t)t * TILE);
            const int ng4 = (nt + 3) >> 2;
            const uint32_t st = seq % NST;
            uint32_t idx = ent & NLN_IDX_MASK, code = ent >> NLN_IDX_BITS;
            // entries are checked at upload, except in the pipelined end-to-end call
            if (lane < nt && (idx >= ntab || code > 26u)) {
                atomicOr(P.err, GC_DEV_BAD_INDEX);
                idx = 0;
                code = NLN_SHIFT_NONE;
            }
            if (lane >= nt)
                idx = 0;
            codes[st * TILE + lane] = code;
            if (lane == 0)
                mbar_arrive_expect_tx(&bar[st], (uint32_t)(ng4 * 4 * RB));
            unsigned char *dst = wbuf + st * K::stage_bytes;
#pragma unroll
            for (int g = 0; g < TILE / 4; g++) {
                const int r0 = __shfl_sync(0xffffffffu, (int)idx, 4 * g);
                const int r1 = __shfl_sync(0xffffffffu, (int)idx, 4 * g + 1);
                const int r2 = __shfl_sync(0xffffffffu, (int)idx, 4 * g + 2);
                const int r3 = __shfl_sync(0xffffffffu, (int)idx, 4 * g + 3);
                if (lane == 0 && g < ng4)
                    tma_gather4(dst + g * K::group_bytes, &tmap, r0, r1, r2, r3, &bar[st]);
            }
        };
        // tiles in flight ahead of the one being computed
        constexpr int AHEAD = PAIRED ? 1 : NST - 1;
#pragma unroll
        for (int p = 0; p < AHEAD; p++)
            if (p < ntile)
                issue(p, fetch(p), tseq + p);
        uint32_t ent_next = fetch(AHEAD);
        for (int t = 0; t < ntile; t++) {
            const uint32_t seq = tseq + t;
            if (!PAIRED) {
                if (t + NST - 1 < ntile)
                    issue(t + NST - 1, ent_next, seq + NST - 1);
                ent_next = fetch(t + NST);
            }
            const int nt = (int)min((int64_t)TILE, nent - (int64_t)t * TILE);
            const uint32_t st = seq % NST;
            bool ok = mbar_wait_bounded(&bar[st], (seq / NST) & 1, P.err);
            if (!__all_sync(0xffffffffu, ok)) {
                // give the copies still in flight a bounded chance to land
                for (int u = t + 1; u < ntile && u < t + NST; u++)
                    mbar_wait_bounded(&bar[(tseq + u) % NST], ((tseq + u) / NST) & 1, P.err,
                                      1u << 10);
                alive = false;
                break;
            }
            unsigned char *bt = wbuf + st * K::stage_bytes;
            Acc4 a{0.f, 0.f, 0.f, 0.f};
            if constexpr (PAIRED) {
                relay_pairs<KIND>(bt, codes[st * TILE + lane], lane < nt, c, P.box, pbuf, lane);
                __syncwarp();  // the stage is free: start the next copy, then compute
                if (t + 1 < ntile)
                    issue(t + 1, ent_next, seq + 1);
                ent_next = fetch(t + 2);
                const float2 nsx = splat2(-ux), nsy = splat2(-uy), nsz = splat2(-uz);
                const float2 e2 = splat2(P.eps2), nqsh = splat2(-P.qsh);
                Acc2h A{splat2(0.f), splat2(0.f), splat2(0.f), splat2(0.f)};
                const int npair = (nt + 1) >> 1;
                auto pair = [&](int q) {
                    if (KIND == KH)
                        hexa2_plummer(pbuf + q * K::pair_stride, nsx, nsy, nsz, e2, nqsh, A);
                    else
                        quad2_plummer(pbuf + q * K::pair_stride, nsx, nsy, nsz, e2, nqsh, A);
                };
                constexpr int kUnroll = KIND == KH ? kH2Unroll : kQ2Unroll;
                if (npair == TILE / 2) {
#pragma unroll kUnroll
                    for (int q = 0; q < TILE / 2; q++) pair(q);
                } else {
                    for (int q = 0; q < npair; q++) pair(q);
                }
                a.ax = A.ax.x + A.ax.y;
                a.ay = A.ay.x + A.ay.y;
                a.az = A.az.x + A.az.y;
                a.phi = -(A.nphi.x + A.nphi.y);
            } else {
            if (lane < nt)
                convert<KIND, STAGED>(bt + K::rec_off(lane), codes[st * TILE + lane], c, P.box);
            __syncwarp();
            if (nt == TILE) {
#pragma unroll 4
                for (int r = 0; r < TILE; r++)
                    interact<ORDER, SOFT_PLUMMER>(reinterpret_cast<const float *>(bt + K::rec_off(r)),
                                                  ux, uy, uz, P.eps2, P.qsh, a);
            } else {
                for (int r = 0; r < nt; r++)
                    interact<ORDER, SOFT_PLUMMER>(reinterpret_cast<const float *>(bt + K::rec_off(r)),
                                                  ux, uy, uz, P.eps2, P.qsh, a);
            }
            }
            if (PLAIN) {
                hi[0] += a.ax;
                hi[1] += a.ay;
                hi[2] += a.az;
                hi[3] += a.phi;
            } else {
                comp_add(hi[0], lo[0], a.ax);
                comp_add(hi[1], lo[1], a.ay);
                comp_add(hi[2], lo[2], a.az);
                comp_add(hi[3], lo[3], a.phi);
            }
            __syncwarp();  // every lane is done with this stage before it is refilled
        }
        tseq += ntile;
        if (!alive)
            break;
        float4 *dst = P.part + ((size_t)item.slot * 32 + lane) * 2;
        dst[0] = make_float4(hi[0], hi[1], hi[2], hi[3]);
        dst[1] = make_float4(lo[0], lo[1], lo[2], lo[3]);
    }
}

// Point records (bodies and cell monopoles, 16 B each) are staged without
// TMA: every lane loads its own record with a plain read-only load, one tile
// ahead of use (the list entry two tiles ahead), re-centres it in registers
// and writes it to the warp's shared tile; the row-gather path costs more
// than it saves for records this small.  The tile is laid out in record
// pairs, field by field (pair j: npx0 npx1 npy0 npy1 | npz0 npz1 m0 m1, with
// np the negated offset), so that each 16-byte shared read yields two ready
// operand pairs for the paired FP32 instructions of mono2_plummer.
template <bool PLAIN = false>
__global__ void __launch_bounds__(256) k_points(DevProblem P) {
    __shared__ __align__(16) float stile[8][TILE * 4];
    const int lane = threadIdx.x & 31;
    float *tile = stile[threadIdx.x >> 5];
    const float4 *tile4 = reinterpret_cast<const float4 *>(tile);
    // this lane's record slot in the pair layout
    float *mine = tile + (lane >> 1) * 8 + (lane & 1);
    const uint32_t *list = P.list[KP];
    const uint32_t ntab = (uint32_t)P.ntab[KP];
    const uint32_t nb = ntab - (uint32_t)P.ncells;
    const bool periodic = P.box > 0;
    const float2 e2 = make_float2(P.eps2, P.eps2);
    while (true) {
        int it = 0;
        if (lane == 0)
            it = atomicAdd(&P.counters[KP], 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= P.nitems[KP])
            break;
        const Item item = P.items[KP][it];
        const nln_group G = P.groups[item.group];
        const double c[3] = {PLAIN ? 0.0 : G.cen[0], PLAIN ? 0.0 : G.cen[1],
                             PLAIN ? 0.0 : G.cen[2]};
        float ux = 0.f, uy = 0.f, uz = 0.f;
        if (lane < G.count) {
            float4 sk = P.points[G.first + lane];
            ux = (float)((double)sk.x - c[0]);
            uy = (float)((double)sk.y - c[1]);
            uz = (float)((double)sk.z - c[2]);
        }
        const float2 sx = make_float2(ux, ux), sy = make_float2(uy, uy), sz = make_float2(uz, uz);
        float hi[4] = {0.f, 0.f, 0.f, 0.f}, lo[4] = {0.f, 0.f, 0.f, 0.f};
        const int64_t nent = item.end - item.begin;
        const int ntile = (int)((nent + TILE - 1) / TILE);
        constexpr uint32_t kNone = 0xffffffffu;  // no entry in this lane
        auto entry = [&](int t) -> uint32_t {
            const int64_t k = item.begin + (int64_t)t * TILE + lane;
            return (t < ntile && k < item.end) ? __ldg(list + k) : kNone;
        };
        // a record's position (FP64: a cell monopole's centre from the staged
        // cell table in the mixed form) and mass
        struct Rec {
            double x, y, z;
            float m;
        };
        auto record = [&](uint32_t &e) -> Rec {
            if (e == kNone)
                return Rec{0.0, 0.0, 0.0, 0.f};
            uint32_t idx = e & NLN_IDX_MASK;
            // entries are checked at upload, except in the pipelined end-to-end call
            if (idx >= ntab || (e >> NLN_IDX_BITS) > 26u) {
                atomicOr(P.err, GC_DEV_BAD_INDEX);
                idx = 0;
                e = NLN_SHIFT_NONE << NLN_IDX_BITS;
            }
            const float4 p = __ldg(P.points + idx);
            if (!PLAIN && P.cstage && idx >= nb) {
                const float4 *cs = P.cstage + (size_t)(idx - nb) * P.cstride;
                const float4 a = __ldg(cs), b = __ldg(cs + 2);
                return Rec{__hiloint2double(__float_as_int(a.y), __float_as_int(a.x)),
                           __hiloint2double(__float_as_int(a.w), __float_as_int(a.z)),
                           __hiloint2double(__float_as_int(b.w), __float_as_int(b.z)), p.w};
            }
            return Rec{(double)p.x, (double)p.y, (double)p.z, p.w};
        };
        uint32_t e_cur = entry(0);
        Rec r_cur = record(e_cur);
        uint32_t e_nxt = entry(1);
        for (int t = 0; t < ntile; t++) {
            const Rec r_nxt = record(e_nxt);  // consumed next tile
            const uint32_t e_nn = entry(t + 2);
            const int nt = (int)min((int64_t)TILE, nent - (int64_t)t * TILE);
            // an absent record: massless and far from every sink
            float npx = -1.0e3f, npy = -1.0e3f, npz = -1.0e3f, m = 0.f;
            if (e_cur != kNone) {
                double sxs = 0.0, sys = 0.0, szs = 0.0;
                if (periodic)
                    decode_shift(e_cur >> NLN_IDX_BITS, P.box, sxs, sys, szs);
                npx = (float)(c[0] - (r_cur.x + sxs));
                npy = (float)(c[1] - (r_cur.y + sys));
                npz = (float)(c[2] - (r_cur.z + szs));
                m = r_cur.m;
            }
            __syncwarp();  // the previous tile is no longer read
            mine[0] = npx;
            mine[2] = npy;
            mine[4] = npz;
            mine[6] = m;
            __syncwarp();
            Acc2 a2{make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f),
                    make_float2(0.f, 0.f)};
            if (nt == TILE) {
#pragma unroll 8
                for (int j = 0; j < TILE / 2; j++) {
                    const float4 A = tile4[2 * j], B = tile4[2 * j + 1];
                    mono2_plummer(make_float2(A.x, A.y), make_float2(A.z, A.w),
                                  make_float2(B.x, B.y), make_float2(B.z, B.w), sx, sy, sz, e2, a2);
                }
            } else {
                for (int j = 0; j < (nt + 1) / 2; j++) {
                    const float4 A = tile4[2 * j], B = tile4[2 * j + 1];
                    mono2_plummer(make_float2(A.x, A.y), make_float2(A.z, A.w),
                                  make_float2(B.x, B.y), make_float2(B.z, B.w), sx, sy, sz, e2, a2);
                }
            }
            if (PLAIN) {
                hi[0] -= a2.nax.x + a2.nax.y;
                hi[1] -= a2.nay.x + a2.nay.y;
                hi[2] -= a2.naz.x + a2.naz.y;
                hi[3] -= a2.nphi.x + a2.nphi.y;
            } else {
                comp_add(hi[0], lo[0], -(a2.nax.x + a2.nax.y));
                comp_add(hi[1], lo[1], -(a2.nay.x + a2.nay.y));
                comp_add(hi[2], lo[2], -(a2.naz.x + a2.naz.y));
                comp_add(hi[3], lo[3], -(a2.nphi.x + a2.nphi.y));
            }
            e_cur = e_nxt;
            r_cur = r_nxt;
            e_nxt = e_nn;
        }
        float4 *dst = P.part + ((size_t)item.slot * 32 + lane) * 2;
        dst[0] = make_float4(hi[0], hi[1], hi[2], hi[3]);
        dst[1] = make_float4(lo[0], lo[1], lo[2], lo[3]);
    }
}

// Periodic correction moments (ewald.cuh) of groups gbegin..ngroups-1, one
// warp per group from a queue (counter 3), lanes striding the group's
// correction list, stored per group for k_finish.  Bodies count as masses; a
// cell adds its traceless second to fourth moments (the list's cells
// include coarse ones standing for whole subtrees, and cells a tenth of the
// box wide near the half-box, where C varies on the scale of the cell), and
// its second-moment trace B2/3 against the constant Laplacian of C.
//
// The loads are what bound this loop: each entry needs its table node
// (224 B) and its cell record (128 B) from scattered addresses, and the node
// depends on the record's centre.  So every lane runs a three-deep pipeline
// of its own entries: list word three tiles ahead, the source's FP64 centre
// (a plain load) two tiles ahead, and one tile ahead a per-lane cp.async of
// the node and the record into this warp's shared-memory stage, laid out
// chunk-major ([chunk][lane] float4) so that the compute's reads are
// conflict-free.  Each lane reads only what it copied itself.
constexpr int kEwNodeChunks = 14;  // 56 floats: C and its derivatives of orders 0..5
constexpr int kEwRecChunks = 7;    // floats 4..31 of an order-4 cell record (nln_hcell); the
                                   // centre in floats 0..5 comes with the pipeline's registers
struct EwStage {
    float4 node[kEwNodeChunks][32];
    float4 rec[kEwRecChunks][32];
};
constexpr int kEwWarpBytes = 2 * (int)sizeof(EwStage);  // two stages per warp: 21,504 B

__global__ void __launch_bounds__(128) k_ewald_moments(DevProblem P) {
    extern __shared__ __align__(16) unsigned char ewsm[];
    const int lane = threadIdx.x & 31;
    EwStage *stg = reinterpret_cast<EwStage *>(ewsm + (size_t)(threadIdx.x >> 5) * kEwWarpBytes);
    const uint32_t ntab = (uint32_t)P.ntab[0];
    const uint32_t nb = ntab - (uint32_t)P.ncells;
    constexpr uint32_t kNone = 0xffffffffu;
    // one source of the pipeline: list word (kNone: no entry in this lane)
    // and its position (FP64) with, for a body, its mass
    struct Src {
        uint32_t e;
        double x, y, z;
        float m;
    };
    for (;;) {
        int it = 0;
        if (lane == 0)
            it = atomicAdd(&P.counters[3], 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        const int64_t g = P.gbegin + it;
        if (g >= P.ngroups)
            break;
        const nln_group G = P.groups[g];
        const double c[3] = {G.cen[0], G.cen[1], G.cen[2]};
        const int64_t cb = P.cptr[g], ce = P.cptr[g + 1];
        const int ntile = (int)((ce - cb + 31) / 32);
        // the list word is checked where it is used, a tile after its load
        auto entry = [&](int t) -> uint32_t {
            const int64_t k = cb + (int64_t)t * 32 + lane;
            return (t < ntile && k < ce) ? __ldg(P.clist + k) : kNone;
        };
        auto source = [&](uint32_t e) -> Src {
            Src r{kNone, 0.0, 0.0, 0.0, 0.f};
            if (e == kNone)
                return r;
            const uint32_t idx = e & NLN_IDX_MASK;
            if (idx >= ntab || (e >> NLN_IDX_BITS) > 26u) {  // as in k_batch
                atomicOr(P.err, GC_DEV_BAD_INDEX);
                return r;
            }
            r.e = e;
            if (idx < nb) {
                const float4 p = __ldg(P.points + idx);
                r.x = p.x;
                r.y = p.y;
                r.z = p.z;
                r.m = p.w;
            } else {
                const double *cen = P.hcells[idx - nb].cen;
                r.x = __ldg(cen);
                r.y = __ldg(cen + 1);
                r.z = __ldg(cen + 2);
            }
            return r;
        };
        auto node_of = [&](const Src &q) -> EwNode {
            double sx, sy, sz;
            decode_shift(q.e >> NLN_IDX_BITS, P.box, sx, sy, sz);
            return ew_node(P.ew, (float)(q.x + sx - c[0]), (float)(q.y + sy - c[1]),
                           (float)(q.z + sz - c[2]));
        };
        auto issue = [&](const Src &q, EwStage &S) {
            if (q.e == kNone)
                return;
            const uint32_t idx = q.e & NLN_IDX_MASK;
            const float4 *node =
                reinterpret_cast<const float4 *>(P.ew.t + (size_t)node_of(q).node * ew::kNode);
#pragma unroll
            for (int k = 0; k < kEwNodeChunks; k++) cp_async16(&S.node[k][lane], node + k);
            if (idx >= nb) {
                const float4 *rec = reinterpret_cast<const float4 *>(P.hcells + (idx - nb)) + 1;
#pragma unroll
                for (int k = 0; k < kEwRecChunks; k++) cp_async16(&S.rec[k][lane], rec + k);
            }
        };
        EwMoments M;
        M.zero();
        Src s0 = source(entry(0));
        issue(s0, stg[0]);
        cp_async_commit();
        Src s1 = source(entry(1));
        uint32_t e2 = entry(2);
        for (int t = 0; t < ntile; t++) {
            if (t + 1 < ntile)
                issue(s1, stg[(t + 1) & 1]);
            cp_async_commit();
            const Src s2 = source(e2);  // consumed by the next tile's issue
            e2 = entry(t + 3);
            cp_async_wait<1>();  // this lane's copies for tile t have landed
            if (s0.e != kNone) {
                const EwStage &S = stg[t & 1];
                const EwNode N = node_of(s0);
                // orders 0..4 (35 values) for the expansion; order 5 is read
                // after it, so the two are never in registers together
                float V[36];
#pragma unroll
                for (int k = 0; k < 9; k++) {
                    const float4 v = S.node[k][lane];
                    V[4 * k] = v.x;
                    V[4 * k + 1] = v.y;
                    V[4 * k + 2] = v.z;
                    V[4 * k + 3] = v.w;
                }
                float o[ew::kNQ4], f5[21];
                ew_expand<false>(V, N, o, nullptr);
                if ((s0.e & NLN_IDX_MASK) < nb) {
                    ew_add_mass(M, s0.m, o);
                } else {
                    float V5[24];  // node floats 32..55; order 5 starts at 35
#pragma unroll
                    for (int k = 8; k < kEwNodeChunks; k++) {
                        const float4 v = S.node[k][lane];
                        V5[4 * (k - 8)] = v.x;
                        V5[4 * (k - 8) + 1] = v.y;
                        V5[4 * (k - 8) + 2] = v.z;
                        V5[4 * (k - 8) + 3] = v.w;
                    }
                    ew_fifth(V5 + 3, N, f5);
                    float r[32];
#pragma unroll
                    for (int k = 0; k < kEwRecChunks; k++) {
                        const float4 v = S.rec[k][lane];
                        r[4 * (k + 1)] = v.x;
                        r[4 * (k + 1) + 1] = v.y;
                        r[4 * (k + 1) + 2] = v.z;
                        r[4 * (k + 1) + 3] = v.w;
                    }
                    // nln_hcell floats: mass 6, R 7, q2 8..12, q3 13..19, q4 20..28, B2 29
                    const float R = r[7];
                    ew_add_mass(M, r[6], o);
                    float Sm[15];
                    ew_quad(R, r + 8, Sm);
                    ew_fold<2, 3>(M, Sm, o, f5);
                    ew_oct(R, r + 13, Sm);
                    ew_fold<3, 2>(M, Sm, o, f5);
                    ew_hex(R, r + 20, Sm);
                    ew_fold<4, 1>(M, Sm, o, f5);
                    M.add(0, __fmul_rn(__fmul_rn(r[29], 1.f / 6.f), P.ew_trace));
                }
                M.end_entry();
            }
            s0 = s1;
            s1 = s2;
        }
        cp_async_wait<0>();
        M.warp_sum();
        if (lane == 0) {
            EwStored &E = P.ewm[g];
#pragma unroll
            for (int q = 0; q < 10; q++) E.lo[q] = M.lo[q];
#pragma unroll
            for (int q = 0; q < 25; q++) E.hi[q] = M.hi[q];
        }
    }
}

// The same correction moments of group g by a plain loop over the list,
// lanes striding it, every load on demand: no shared memory and fewer
// registers than k_ewald_moments, which suits a kernel that shares the SMs
// with the list kernels (the side stream).  The arithmetic and its order are
// k_ewald_moments', so the two store identical moments.  Bodies count as masses; a cell adds its
// traceless second to fourth moments (the list's cells include coarse
// ones standing for whole subtrees, and cells a tenth of the box wide near
// the half-box, where C varies on the scale of the cell), and its
// second-moment trace B2/3 against the constant Laplacian of C.
__device__ __forceinline__ void ewald_moments_loop(const DevProblem &P, int64_t g, const double *c,
                                              int lane, EwMoments &M) {
    M.zero();
    float o[ew::kNQ4], f5[21];
    const uint32_t nb = (uint32_t)P.ntab[0] - (uint32_t)P.ncells;
    for (int64_t k = P.cptr[g] + lane; k < P.cptr[g + 1]; k += 32) {
        const uint32_t ent = P.clist[k];
        const uint32_t idx = ent & NLN_IDX_MASK;
        if (idx >= (uint32_t)P.ntab[0] || (ent >> NLN_IDX_BITS) > 26u) {  // as in k_batch
            atomicOr(P.err, GC_DEV_BAD_INDEX);
            continue;
        }
        double sx, sy, sz;
        decode_shift(ent >> NLN_IDX_BITS, P.box, sx, sy, sz);
        if (idx < nb) {
            const float4 p = P.points[idx];
            ew_lookup<false>(P.ew, (float)((double)p.x + sx - c[0]),
                             (float)((double)p.y + sy - c[1]), (float)((double)p.z + sz - c[2]),
                             o, nullptr);
            ew_add_mass(M, p.w, o);
        } else {
            const nln_hcell &h = P.hcells[idx - nb];
            ew_lookup<true>(P.ew, (float)(h.cen[0] + sx - c[0]), (float)(h.cen[1] + sy - c[1]),
                            (float)(h.cen[2] + sz - c[2]), o, f5);
            ew_add_mass(M, h.mass, o);
            float S[15];
            ew_quad(h.R, h.q2, S);
            ew_fold<2, 3>(M, S, o, f5);
            ew_oct(h.R, h.q3, S);
            ew_fold<3, 2>(M, S, o, f5);
            ew_hex(h.R, h.q4, S);
            ew_fold<4, 1>(M, S, o, f5);
            M.add(0, __fmul_rn(__fmul_rn(h.B2, 1.f / 6.f), P.ew_trace));
        }
        M.end_entry();
    }
    M.warp_sum();
}

// The correction moments of groups gbegin..ngroups-1 by ewald_moments_loop,
// stored per group for k_finish: one warp per group from a queue (counter
// 3), run on a side stream beside the list kernels, which it does not
// depend on.
__global__ void __launch_bounds__(64) k_ewald_side(DevProblem P) {
    const int lane = threadIdx.x & 31;
    for (;;) {
        int it = 0;
        if (lane == 0)
            it = atomicAdd(&P.counters[3], 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        const int64_t g = P.gbegin + it;
        if (g >= P.ngroups)
            break;
        const nln_group G = P.groups[g];
        const double c[3] = {G.cen[0], G.cen[1], G.cen[2]};
        EwMoments M;
        ewald_moments_loop(P, g, c, lane, M);
        if (lane == 0) {
            EwStored &E = P.ewm[g];
#pragma unroll
            for (int q = 0; q < 10; q++) E.lo[q] = M.lo[q];
#pragma unroll
            for (int q = 0; q < 25; q++) E.hi[q] = M.hi[q];
        }
    }
}

// Per group, in slot order: sum the partials of its work items in FP64,
// add the periodic correction, and write (ax, ay, az, phi) of each sink.
__global__ void k_finish(DevProblem P) {
    const int64_t g = P.gbegin + (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (g >= P.ngroups)
        return;
    const nln_group G = P.groups[g];
    double s[4] = {0, 0, 0, 0};
    for (int64_t k = P.gslot[g]; k < P.gslot[g + 1]; k++) {
        const float4 *src = P.part + ((size_t)k * 32 + lane) * 2;
        float4 h = src[0], l = src[1];
        s[0] += (double)h.x + (double)l.x;
        s[1] += (double)h.y + (double)l.y;
        s[2] += (double)h.z + (double)l.z;
        s[3] += (double)h.w + (double)l.w;
    }
    if (P.ewald) {
        const double c[3] = {G.cen[0], G.cen[1], G.cen[2]};
        EwMoments M;
        const EwStored &E = P.ewm[g];  // k_ewald_moments
#pragma unroll
        for (int q = 0; q < 10; q++) M.lo[q] = E.lo[q];
#pragma unroll
        for (int q = 0; q < 25; q++) M.hi[q] = E.hi[q];
        if (lane < G.count) {
            const float4 p = P.points[G.first + lane];
            double phi, ax, ay, az;
            ew_apply(M, (double)p.x - c[0], (double)p.y - c[1], (double)p.z - c[2], phi, ax, ay,
                     az);
            s[0] += ax;
            s[1] += ay;
            s[2] += az;
            s[3] += phi - (double)p.w * P.ew_self;
        }
    }
    if (lane < G.count)
        P.out[G.first + lane] = make_float4((float)s[0], (float)s[1], (float)s[2], (float)s[3]);
}

}  // namespace

// ------------------------------------------------------------ plan
struct grav_step_state;  // time-step state (step.cuh)
void step_state_free(grav_step_state *S);
void step_graph_reset(grav_step_state *S);
struct grav_adjoint_state;  // adjoint scratch (adjoint.cuh)
void adjoint_state_free(grav_adjoint_state *A);

struct grav_plan {
    grav_problem hp{};      // sizes and parameters (host pointers cleared)
    grav_tuning tune{};
    DevProblem dp{};
    std::vector<void *> allocs;
    int64_t counts[4] = {0, 0, 0, 0};
    int nsm = 148;
    int launches = 0;
    int64_t nslots = 0;
    CUtensorMap tmap[3];    // row-gather views of the point, quadrupole and order-4 tables
    int timing = 0;         // record events around each kernel of an evaluation
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    std::vector<int64_t> lists_ptr[4];  // host copies of the P, Q, H (queue rebuilds) and
                                        // correction list offsets
    int64_t *order = nullptr;           // device-built plans: tree position -> input index
    bool staged = false;                // the Q/H tensor maps view pre-staged tables
    bool plain = false;                 // plain FP32 kernels (grav_problem.precision = 1)
    int integrator = 0;                 // 0: Integrate, 1: CosmoIntegrate (step.cuh)
    bool evaluated = false;             // grav_groups_eval_CUDA has been enqueued (the
                                        // correction moments the adjoint reads are set)
    float4 *qstage = nullptr, *hstage = nullptr;  // pre-staged cell tables (k_stage_cells)
    grav_step_state *step = nullptr;  // tree links, refit scratch and the step graph
    grav_adjoint_state *adj = nullptr;  // adjoint scratch
    // periodic: the side stream of k_ewald_moments, its fork/join events and
    // the per-group correction moments
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    EwStored *ewm = nullptr;
    int64_t ewald_entries = 0;  // correction-list length
    // Group ranges of the work queue: items are sorted by cost within each
    // range, and chunk_item[k][c] is the first item of kind k in range c.
    // One range [0, ngroups) except in the pipelined end-to-end call.
    std::vector<int64_t> chunk_group;
    std::vector<int> chunk_item[3];
    cudaMemPool_t pool = nullptr;  // device buffers from this pool (the end-to-end call)
    // run-packed lists of the end-to-end call (P, Q, H, correction): device
    // words, their offsets and the plain offsets they unpack to
    uint32_t *zdev[4] = {nullptr, nullptr, nullptr, nullptr};
    const int64_t *zptr_dev[4] = {nullptr, nullptr, nullptr, nullptr};
    const int64_t *lptr_dev[4] = {nullptr, nullptr, nullptr, nullptr};
};

namespace {

// A 2-D tensor map over `rows` records of `row_bytes` (a multiple of 16),
// box = one full record (one row high, as the row gather requires).
int encode_rows(CUtensorMap *m, const void *base, uint64_t rows, uint32_t row_bytes) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        GC_CHECK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        if (!fn || q != cudaDriverEntryPointSuccess)
            return gc::set_status(-1, "cuTensorMapEncodeTiled unavailable");
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    const uint32_t w = row_bytes / 4;
    cuuint64_t dims[2] = {w, rows};
    cuuint64_t strides[1] = {row_bytes};
    cuuint32_t box[2] = {w, 1};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void *>(base), dims,
                        strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return gc::set_status(-1, "cuTensorMapEncodeTiled failed (%d) for %llu rows of %u bytes",
                              (int)r, (unsigned long long)rows, row_bytes);
    return 0;
}

template <typename T>
int dev_copy(grav_plan *pl, const T *src, size_t n, T **dst);

// dev_copy whose copy is asynchronous on the default stream when `async`
// (the end-to-end call's pool allocations are ordered on that stream).
template <typename T>
int dev_copy(grav_plan *pl, bool async, const T *src, size_t n, T **dst) {
    if (!async || !pl->pool)
        return dev_copy(pl, src, n, dst);
    if (int rc = dev_copy<T>(pl, nullptr, n, dst))
        return rc;
    if (src && n)
        GC_CHECK(cudaMemcpyAsync(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice, 0));
    return 0;
}

template <typename T>
int dev_copy(grav_plan *pl, const T *src, size_t n, T **dst) {
    *dst = nullptr;
    if (n == 0)
        return 0;
    if (pl->pool) {
        if (cudaMallocFromPoolAsync((void **)dst, n * sizeof(T), pl->pool, 0) != cudaSuccess) {
            // the pool's reserved but unused memory may be what is missing
            cudaGetLastError();
            cudaStreamSynchronize(0);
            cudaMemPoolTrimTo(pl->pool, 0);
            GC_CHECK(cudaMallocFromPoolAsync((void **)dst, n * sizeof(T), pl->pool, 0));
        }
    } else
        GC_CHECK(cudaMalloc((void **)dst, n * sizeof(T)));
    pl->allocs.push_back(*dst);
    if (src)
        GC_CHECK(cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice));
    return 0;
}

// Defaults: 8 warps per block, as many resident blocks as registers and
// shared memory allow (blocks_per_sm = 0), list chunks sized automatically
// (chunk_* = 0) from the totals once the lists are known.
grav_tuning default_tuning() {
    grav_tuning t;
    t.warps_per_block = 8;
    t.blocks_per_sm = 0;
    t.chunk_p = t.chunk_q = t.chunk_h = 0;
    t.ewald_n = 0;
    t.ewald_side = 0;
    return t;
}

// Split lists so that there are at least ~8 work items per resident warp
// (about 148 SMs x 32 warps), in whole tiles, no shorter than `lo`.
int auto_chunk(int64_t total, int64_t ngroups, int nsm, int64_t lo) {
    const int64_t warps = (int64_t)nsm * 32;
    int64_t ng = std::max<int64_t>(ngroups, 1);
    int64_t per = std::max<int64_t>(1, (8 * warps + ng - 1) / ng);
    int64_t avg = std::max<int64_t>(1, total / ng);
    int64_t c = std::max<int64_t>(lo, avg / per);
    c = (c + TILE - 1) / TILE * TILE;
    return (int)std::min<int64_t>(1 << 24, c);
}

// Work items of a plan from its kept list offsets and tuning: created group
// by group (slot order: a group's point items, then quadrupole, then order 4),
// then ordered per kind by cost, longest first, within each of the plan's
// group ranges (chunk_group; the whole set when empty).  Every item but a
// group's last of a kind is a full chunk, so the order is the full chunks in
// creation order, then the remainders by length (both stable).
int64_t make_queue(grav_plan *pl, std::vector<Item> items[3], std::vector<int64_t> &gslot) {
    const int64_t ng = pl->hp.ngroups;
    const int64_t chunk[3] = {pl->tune.chunk_p, pl->tune.chunk_q, pl->tune.chunk_h};
    if (pl->chunk_group.size() < 2)
        pl->chunk_group = {0, ng};
    const int nc = (int)pl->chunk_group.size() - 1;
    const int64_t *ptr[3];
    for (int k = 0; k < 3; k++) ptr[k] = pl->lists_ptr[k].empty() ? nullptr : pl->lists_ptr[k].data();
    // items per group and kind, then their first index and slot by prefix sums
    std::vector<int64_t> first[3];
    for (int k = 0; k < 3; k++) first[k].assign(ng + 1, 0);
    gslot.assign(ng + 1, 0);
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < ng; g++) {
        int64_t all = 0;
        for (int k = 0; k < 3; k++) {
            const int64_t n = ptr[k] ? (ptr[k][g + 1] - ptr[k][g] + chunk[k] - 1) / chunk[k] : 0;
            first[k][g + 1] = n;
            all += n;
        }
        gslot[g + 1] = all;
    }
    for (int64_t g = 0; g < ng; g++) {
        for (int k = 0; k < 3; k++) first[k][g + 1] += first[k][g];
        gslot[g + 1] += gslot[g];
    }
    for (int k = 0; k < 3; k++) items[k].resize((size_t)first[k][ng]);
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < ng; g++) {
        int32_t slot = (int32_t)gslot[g];
        for (int k = 0; k < 3; k++) {
            if (!ptr[k])
                continue;
            Item *out = items[k].data() + first[k][g];
            for (int64_t b = ptr[k][g]; b < ptr[k][g + 1]; b += chunk[k])
                *out++ = Item{(int32_t)g, slot++, b, std::min(ptr[k][g + 1], b + chunk[k])};
        }
    }
    for (int k = 0; k < 3; k++) {
        pl->chunk_item[k].resize(nc + 1);
        for (int c = 0; c <= nc; c++) pl->chunk_item[k][c] = (int)first[k][pl->chunk_group[c]];
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int task = 0; task < 3 * nc; task++) {
        const int k = task % 3, c = task / 3;
        auto b = items[k].begin() + pl->chunk_item[k][c], e = items[k].begin() + pl->chunk_item[k][c + 1];
        const int64_t full = chunk[k];
        auto mid = std::stable_partition(b, e, [full](const Item &x) { return x.end - x.begin == full; });
        std::stable_sort(mid, e, [](const Item &x, const Item &y) {
            return (x.end - x.begin) > (y.end - y.begin);
        });
    }
    return gslot[ng];
}

// The device address of page-locked host memory (lists read in place over
// PCIe), or null when `p` is not page-locked host memory.
const uint32_t *mapped_host(const uint32_t *p) {
    cudaPointerAttributes a{};
    if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return a.type == cudaMemoryTypeHost ? static_cast<const uint32_t *>(a.devicePointer) : nullptr;
}

}  // namespace

namespace {
// The upload.  With nchunks > 0 (the pipelined end-to-end call) the list
// buffers are allocated but not filled: the caller copies each group range's
// lists while the kernels evaluate the previous range, and the kernels'
// own index checks stand in for the upload-time list check.
thread_local double t_phase[5];  // grav_groups_CUDA_phases
thread_local double t_build = 0, t_build_phase[6] = {0, 0, 0, 0, 0, 0};  // grav_plan_build_phases
thread_local double t_phase_be[4] = {0, 0, 0, 0};  // grav_build_eval_phases

// The end-to-end call's device buffers come from a pool per device that
// keeps freed memory reserved (until grav_groups_release_CUDA): mapping and
// unmapping tens of gigabytes in every call costs as much as the
// evaluation's tail.
constexpr int kMaxPoolDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[kMaxPoolDevices] = {};

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

int e2e_pool(cudaMemPool_t *out) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    int dev = 0;
    GC_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxPoolDevices)
        return gc::set_status(-1, "grav_groups_CUDA: device %d beyond %d", dev, kMaxPoolDevices);
    if (!g_pool[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        GC_CHECK(cudaMemPoolCreate(&g_pool[dev], &props));
        uint64_t keep = UINT64_MAX;
        GC_CHECK(cudaMemPoolSetAttribute(g_pool[dev], cudaMemPoolAttrReleaseThreshold, &keep));
    }
    *out = g_pool[dev];
    return 0;
}

// adopt: a tree built on the device (gpu_tree_build) whose tables and lists
// the plan takes over instead of copying; hp then holds its host copies of
// the groups and offsets and device pointers to everything else.
int upload_impl(const grav_problem *hp, const grav_tuning *tuning, grav_plan **plan_out,
                int nchunks, const DevTree *adopt = nullptr) {
    *plan_out = nullptr;
    const double t_start = now_s();
    if (!hp || hp->nbodies <= 0 || hp->ngroups <= 0 || !hp->points || !hp->groups ||
        !hp->pptr || (!hp->plist && !(nchunks > 0 && hp->zlist[0])))
        return gc::set_status(-1, "grav_groups_upload_CUDA: incomplete problem");
    if (hp->nbodies + hp->ncells >= (int64_t)NLN_IDX_MASK)
        return gc::set_status(-1, "grav_groups_upload_CUDA: point table exceeds 27-bit indices");
    if (hp->precision != 0 && hp->precision != 1)
        return gc::set_status(-1, "grav_groups_upload_CUDA: precision must be 0 (mixed) or 1 "
                                  "(plain FP32)");
    grav_plan *pl = new grav_plan();
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&pl->nsm, cudaDevAttrMultiProcessorCount, dev);
    pl->hp = *hp;
    pl->plain = hp->precision == 1;
    if (adopt) {
        pl->pool = adopt->pool;  // freed the way they were allocated
        // the plan owns every buffer of the device-built tree from here on,
        // failures included (grav_plan_free releases them)
        void *own[] = {adopt->points, adopt->qcells, adopt->hcells, adopt->groups,
                       adopt->list[0], adopt->list[1], adopt->list[2], adopt->list[3],
                       adopt->order};
        for (void *q : own)
            if (q)
                pl->allocs.push_back(q);
        pl->order = adopt->order;
    }
    pl->tune = tuning ? *tuning : default_tuning();
    const int64_t ng = hp->ngroups, nb = hp->nbodies, np = hp->nbodies + hp->ncells;
    const bool deferred = nchunks > 0;
    if (deferred && hp->lists_in_host) {
        grav_plan_free(pl);
        return gc::set_status(-1, "upload: deferred lists and lists_in_host exclude each other");
    }
    if (deferred) {
        if (int e = e2e_pool(&pl->pool)) {
            grav_plan_free(pl);
            return e;
        }
    }

    // validate everything the kernels will index
    int bad_group = 0;
#pragma omp parallel for schedule(static) reduction(| : bad_group)
    for (int64_t g = 0; g < ng; g++) {
        const nln_group &G = hp->groups[g];
        if (G.count < 1 || G.count > 32 || G.first < 0 || G.first + G.count > nb)
            bad_group |= 1;
        if (hp->pptr[g + 1] < hp->pptr[g] || (hp->qptr && hp->qptr[g + 1] < hp->qptr[g]) ||
            (hp->hptr && hp->hptr[g + 1] < hp->hptr[g]))
            bad_group |= 1;
    }
    if (hp->pptr[0] != 0 || (hp->qptr && hp->qptr[0] != 0) || (hp->hptr && hp->hptr[0] != 0))
        bad_group |= 1;
    if (bad_group) {
        grav_plan_free(pl);
        return gc::set_status(-1, "a group has 0 or more than 32 sinks, lies outside the bodies, "
                                  "or has list offsets that decrease or do not start at 0");
    }
    // Every list entry is checked on the device: after the upload (k_check_lists),
    // or by the kernels as they read it (deferred lists, lists_in_host).  A host
    // pass over tens of gigabytes of lists would dominate an end-to-end call.
    const int64_t *eptr = hp->pptr;
    if ((hp->qptr && hp->qptr[ng] && (!hp->qcells || hp->ncells <= 0)) ||
        (hp->hptr && hp->hptr[ng] && (!hp->hcells || hp->ncells <= 0))) {
        grav_plan_free(pl);
        return gc::set_status(-1, "a cell list without its cell table");
    }
    const bool want_ewald = hp->box > 0 && hp->ewald;
    if (want_ewald) {
        if (!hp->cptr || (!hp->clist && !(deferred && hp->zlist[3])) ||
            (hp->ncells > 0 && !hp->hcells)) {
            grav_plan_free(pl);
            return gc::set_status(-1, "the Ewald correction needs the correction list and the "
                                      "order-4 cell table");
        }
        int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
        for (int64_t g = 0; g < ng; g++)
            if (hp->cptr[g + 1] < hp->cptr[g])
                bad |= 1;
        if (bad || hp->cptr[0] != 0) {
            grav_plan_free(pl);
            return gc::set_status(-1, "bad correction list offsets");
        }
    }
    // run-packed lists (the end-to-end call): offsets from 0, never decreasing
    const int64_t *plain_ptr[4] = {hp->pptr, hp->qptr, hp->hptr, want_ewald ? hp->cptr : nullptr};
    bool packed[4] = {false, false, false, false};
    if (deferred) {
        for (int k = 0; k < 4; k++) {
            if (!hp->zlist[k] || !plain_ptr[k] || plain_ptr[k][ng] == 0)
                continue;
            const int64_t *z = hp->zptr[k];
            int bad = !z || z[0] != 0;
            if (!bad) {
#pragma omp parallel for schedule(static) reduction(| : bad)
                for (int64_t g = 0; g < ng; g++)
                    if (z[g + 1] < z[g])
                        bad |= 1;
            }
            if (bad) {
                grav_plan_free(pl);
                return gc::set_status(-1, "bad run-packed list offsets (kind %d)", k);
            }
            packed[k] = true;
        }
        if (!hp->plist && !packed[0]) {
            grav_plan_free(pl);
            return gc::set_status(-1, "grav_groups_CUDA: no point list");
        }
    }

    // The tables go first: in the end-to-end call (pool allocations, stream
    // ordered) their copies are asynchronous and overlap the work queue's
    // host build below; the upload's later copies and its final
    // synchronisation order everything before the kernels start.
    DevProblem &d = pl->dp;
    int rc = 0;
    float4 *pts = nullptr;
    nln_qcell *qc = nullptr;
    nln_hcell *hc = nullptr;
    nln_group *gr = nullptr;
    const bool want_q = hp->qptr && hp->qptr[ng];
    const bool want_h = (hp->hptr && hp->hptr[ng]) || (want_ewald && hp->ncells > 0);
    if (adopt) {
        pts = adopt->points;
        qc = want_q ? adopt->qcells : nullptr;
        hc = want_h ? adopt->hcells : nullptr;
        gr = adopt->groups;
    } else {
        rc |= dev_copy(pl, deferred, reinterpret_cast<const float4 *>(hp->points), (size_t)np,
                       &pts);
        if (want_q)
            rc |= dev_copy(pl, deferred, hp->qcells, (size_t)hp->ncells, &qc);
        if (want_h)
            rc |= dev_copy(pl, deferred, hp->hcells, (size_t)hp->ncells, &hc);
        rc |= dev_copy(pl, deferred, hp->groups, (size_t)ng, &gr);
    }
    d.points = pts;
    d.qcells = qc;
    d.hcells = hc;
    d.groups = gr;
    if (pl->tune.warps_per_block < 1 || pl->tune.warps_per_block > 8)
        pl->tune.warps_per_block = 8;
    if (pl->tune.chunk_p <= 0)
        pl->tune.chunk_p = auto_chunk(eptr[ng], ng, pl->nsm, 128);
    if (pl->tune.chunk_q <= 0)
        pl->tune.chunk_q = auto_chunk(hp->qptr ? hp->qptr[ng] : 0, ng, pl->nsm, 64);
    if (pl->tune.chunk_h <= 0)
        pl->tune.chunk_h = auto_chunk(hp->hptr ? hp->hptr[ng] : 0, ng, pl->nsm, 32);

    // work items, created group by group (slot order), then sorted per kind by cost
    std::vector<Item> items[3];
    std::vector<int64_t> gslot;
    const int64_t *ptrs[4] = {eptr, hp->qptr, hp->hptr, want_ewald ? hp->cptr : nullptr};
    for (int k = 0; k < 4; k++)
        if (ptrs[k])
            pl->lists_ptr[k].assign(ptrs[k], ptrs[k] + ng + 1);
    if (deferred) {
        // group ranges holding about equal list bytes
        auto bytes_to = [&](int64_t g) {
            int64_t b = eptr[g];
            if (hp->qptr)
                b += hp->qptr[g];
            if (hp->hptr)
                b += hp->hptr[g];
            if (want_ewald)
                b += hp->cptr[g];
            return b;
        };
        // The first range's copy is not overlapped: split it further into
        // 1/8, 1/8, 1/4 and 1/2 of an equal share.
        const int64_t total = std::max<int64_t>(1, bytes_to(ng));
        std::vector<int64_t> wants;
        if (nchunks > 1)
            for (int d : {8, 4, 2}) wants.push_back(total / ((int64_t)nchunks * d));
        for (int c = 1; c < nchunks; c++) wants.push_back(total * c / nchunks);
        pl->chunk_group.assign(1, 0);
        int64_t g = 0;
        for (const int64_t want : wants) {
            int64_t lo = g, hi = ng;  // first group whose prefix reaches `want`
            while (lo < hi) {
                const int64_t mid = (lo + hi) / 2;
                if (bytes_to(mid) < want)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            g = lo;
            if (g > pl->chunk_group.back() && g < ng)
                pl->chunk_group.push_back(g);
        }
        pl->chunk_group.push_back(ng);
    }
    pl->nslots = make_queue(pl, items, gslot);

    // interaction counts (sinks x sources); the point list's split into
    // bodies and cell monopoles is counted on the device (k_check_lists)
    for (int64_t g = 0; g < ng; g++) {
        const int64_t c = hp->groups[g].count;
        if (hp->qptr)
            pl->counts[2] += c * (hp->qptr[g + 1] - hp->qptr[g]);
        if (hp->hptr)
            pl->counts[3] += c * (hp->hptr[g + 1] - hp->hptr[g]);
    }

    t_phase[0] = now_s() - t_start;
    const double t_dev = now_s();
    uint32_t *l0 = nullptr, *l1 = nullptr, *l2 = nullptr, *all_clist = nullptr;
    if (deferred) {
        // one buffer for the four lists, filled range by range by the caller
        const size_t n[4] = {(size_t)hp->pptr[ng], hp->qptr ? (size_t)hp->qptr[ng] : 0,
                             hp->hptr ? (size_t)hp->hptr[ng] : 0,
                             want_ewald ? (size_t)std::max<int64_t>(1, hp->cptr[ng]) : 0};
        size_t off[4], words = 0;
        for (int k = 0; k < 4; k++) {
            off[k] = words;
            words += (n[k] + 63) / 64 * 64;
        }
        uint32_t *all = nullptr;
        rc |= dev_copy<uint32_t>(pl, nullptr, words, &all);
        if (all) {
            l0 = n[0] ? all + off[0] : nullptr;
            l1 = n[1] ? all + off[1] : nullptr;
            l2 = n[2] ? all + off[2] : nullptr;
            all_clist = n[3] ? all + off[3] : nullptr;
        }
        // packed kinds: device words (filled range by range) and both offset arrays
        for (int k = 0; k < 4; k++) {
            if (!packed[k])
                continue;
            uint32_t *zw = nullptr;
            int64_t *zp = nullptr, *lp = nullptr;
            rc |= dev_copy<uint32_t>(pl, nullptr, (size_t)std::max<int64_t>(1, hp->zptr[k][ng]), &zw);
            rc |= dev_copy(pl, hp->zptr[k], (size_t)ng + 1, &zp);
            rc |= dev_copy(pl, plain_ptr[k], (size_t)ng + 1, &lp);
            pl->zdev[k] = zw;
            pl->zptr_dev[k] = zp;
            pl->lptr_dev[k] = lp;
        }
    } else if (adopt) {
        l0 = adopt->list[0];
        l1 = hp->qptr ? adopt->list[1] : nullptr;
        l2 = hp->hptr ? adopt->list[2] : nullptr;
    } else if (hp->lists_in_host) {
        // the kernels read the lists in place from page-locked host memory
        const uint32_t *m0 = mapped_host(hp->plist);
        const uint32_t *m1 = hp->qptr ? mapped_host(hp->qlist) : nullptr;
        const uint32_t *m2 = hp->hptr ? mapped_host(hp->hlist) : nullptr;
        if (!m0 || (hp->qptr && !m1) || (hp->hptr && !m2)) {
            grav_plan_free(pl);
            return gc::set_status(-1, "grav_groups_upload_CUDA: lists_in_host needs the lists in "
                                      "page-locked host memory (cudaHostAlloc)");
        }
        l0 = const_cast<uint32_t *>(m0);
        l1 = const_cast<uint32_t *>(m1);
        l2 = const_cast<uint32_t *>(m2);
    } else {
        rc |= dev_copy(pl, hp->plist, (size_t)hp->pptr[ng], &l0);
        if (hp->qptr)
            rc |= dev_copy(pl, hp->qlist, (size_t)hp->qptr[ng], &l1);
        if (hp->hptr)
            rc |= dev_copy(pl, hp->hlist, (size_t)hp->hptr[ng], &l2);
    }
    d.list[0] = l0;
    d.list[1] = l1;
    d.list[2] = l2;
    d.ntab[0] = np;
    d.ntab[1] = d.ntab[2] = hp->ncells;
    for (int k = 0; k < 3; k++) {
        Item *it = nullptr;
        rc |= dev_copy(pl, items[k].data(), items[k].size(), &it);
        d.items[k] = it;
        d.nitems[k] = (int)items[k].size();
    }
    int *ctr = nullptr;  // 4 queue heads per group range
    rc |= dev_copy<int>(pl, nullptr, 4 * (pl->chunk_group.size() - 1), &ctr);
    d.counters = ctr;
    float4 *part = nullptr;
    rc |= dev_copy<float4>(pl, nullptr, (size_t)std::max<int64_t>(1, pl->nslots) * 64, &part);
    d.part = part;
    int64_t *gs = nullptr;
    rc |= dev_copy(pl, gslot.data(), gslot.size(), &gs);
    d.gslot = gs;
    d.cptr = nullptr;
    d.clist = nullptr;
    if (want_ewald) {
        int64_t *cp = nullptr;
        uint32_t *cl = nullptr;
        rc |= dev_copy(pl, hp->cptr, (size_t)ng + 1, &cp);
        if (hp->lists_in_host) {
            cl = const_cast<uint32_t *>(mapped_host(hp->clist));
            if (!cl) {
                grav_plan_free(pl);
                return gc::set_status(-1, "grav_groups_upload_CUDA: lists_in_host needs the "
                                          "correction list in page-locked host memory");
            }
        } else if (deferred) {
            cl = all_clist;
        } else if (adopt) {
            cl = adopt->list[3];
        } else {
            rc |= dev_copy(pl, hp->clist, (size_t)std::max<int64_t>(1, hp->cptr[ng]), &cl);
        }
        d.cptr = cp;
        d.clist = cl;
    }
    d.ewald = 0;
    if (want_ewald) {
        // FP64 table on the host, FP32 copy on the device
        const int n = pl->tune.ewald_n > 1 ? pl->tune.ewald_n : 32;
        // the table depends only on (box, n): build it once per process
        static std::mutex cache_mu;
        static double cache_box = 0;
        static int cache_n = 0;
        static std::vector<double> t64;
        {
            std::lock_guard<std::mutex> lk(cache_mu);
            if (cache_box != hp->box || cache_n != n) {
                t64.assign((size_t)n * n * n * NLN_EWALD_NQ, 0.0);
                if (ewald_table(hp->box, n, NLN_EWALD_REACH, t64.data())) {
                    grav_plan_free(pl);
                    return gc::set_status(-1, "Ewald table build failed");
                }
                cache_box = hp->box;
                cache_n = n;
            }
        }
        std::vector<float> t32(t64.begin(), t64.end());
        float *tab = nullptr;
        rc |= dev_copy(pl, t32.data(), t32.size(), &tab);
        const double h = NLN_EWALD_REACH * hp->box / (n - 1);
        d.ew = EwTab{tab, n, (float)h, (float)(1.0 / h)};
        const double alpha = 2.0 / hp->box;
        d.ew_self = (float)(t64[0] - M_PI / (alpha * alpha * hp->box * hp->box * hp->box));
        d.ew_trace = (float)(-4.0 * M_PI / (hp->box * hp->box * hp->box));
        d.ewald = 1;
        rc |= dev_copy<EwStored>(pl, nullptr, (size_t)ng, &pl->ewm);
        pl->ewald_entries = hp->cptr[ng];
        cudaError_t e = cudaStreamCreateWithFlags(&pl->side, cudaStreamNonBlocking);
        if (e == cudaSuccess)
            e = cudaEventCreateWithFlags(&pl->fork, cudaEventDisableTiming);
        if (e == cudaSuccess)
            e = cudaEventCreateWithFlags(&pl->join, cudaEventDisableTiming);
        if (e != cudaSuccess)
            rc |= gc::cuda_status(e, "upload: side stream");
    }
    float4 *out = nullptr;
    rc |= dev_copy<float4>(pl, nullptr, (size_t)nb, &out);
    d.out = out;
    unsigned *err = nullptr;
    rc |= dev_copy<unsigned>(pl, nullptr, 1, &err);
    d.err = err;
    if (rc) {
        grav_plan_free(pl);
        return rc;
    }
    cudaMemset(err, 0, sizeof(unsigned));
    if (adopt) {
        // lists from the device builder, which sized and checked them itself
        for (int k = 0; k < 4; k++) pl->counts[k] = adopt->counts[k];
    } else if (hp->lists_in_host || deferred) {
        // entries are checked by the kernels as they read them (bad ones set
        // the error word); the point list's body/cell split is not counted
        int64_t tot = 0;
        for (int64_t g = 0; g < ng; g++) tot += (int64_t)hp->groups[g].count * (hp->pptr[g + 1] - hp->pptr[g]);
        pl->counts[0] = tot;
        pl->counts[1] = 0;
    } else {
        // check every list entry on the device and count the point list's split
        unsigned long long *acc = nullptr;
        rc |= dev_copy<unsigned long long>(pl, nullptr, 3, &acc);
        if (rc) {
            grav_plan_free(pl);
            return rc;
        }
        cudaMemset(acc, 0, 3 * sizeof(unsigned long long));
        const unsigned blocks = (unsigned)pl->nsm * 8;
        const uint32_t ntabs[3] = {(uint32_t)np, (uint32_t)hp->ncells, (uint32_t)hp->ncells};
        for (int k = 0; k < 3; k++)
            if (d.nitems[k] > 0)
                k_check_lists<<<blocks, 256>>>(d.list[k], d.items[k], d.nitems[k], nullptr, 0,
                                                d.groups, ntabs[k], (uint32_t)nb, k == KP, acc);
        if (d.cptr)
            k_check_lists<<<blocks, 256>>>(d.clist, nullptr, 0, d.cptr, ng, d.groups, (uint32_t)np,
                                            (uint32_t)nb, 0, acc);
        unsigned long long h[3] = {0, 0, 0};
        const cudaError_t e = cudaMemcpy(h, acc, sizeof(h), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            grav_plan_free(pl);
            return gc::cuda_status(e, "grav_groups_upload_CUDA: list check");
        }
        if (h[0]) {
            grav_plan_free(pl);
            return gc::set_status(-1, "a list entry lies outside its table or has an image code "
                                      "beyond 26");
        }
        pl->counts[0] = (int64_t)h[1];
        pl->counts[1] = (int64_t)h[2];
    }
    memset(pl->tmap, 0, sizeof(pl->tmap));
    // pre-staged copies of the cell tables the Q and H lists gather from
    if (d.qcells && hp->qptr && hp->qptr[ng])
        rc |= dev_copy<float4>(pl, nullptr, (size_t)hp->ncells * 4, &pl->qstage);
    if (d.hcells && hp->hptr && hp->hptr[ng])
        rc |= dev_copy<float4>(pl, nullptr, (size_t)hp->ncells * 8, &pl->hstage);
    if (!rc && (pl->qstage || pl->hstage)) {
        k_stage_cells<<<(unsigned)((hp->ncells + 127) / 128), 128>>>(d.qcells, d.hcells, hp->ncells,
                                                                       pl->qstage, pl->hstage);
        const cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) {
            grav_plan_free(pl);
            return gc::cuda_status(e, "grav_groups_upload_CUDA: staging the cell tables");
        }
        pl->staged = true;
    }
    d.cstage = pl->qstage ? pl->qstage : pl->hstage;
    d.cstride = pl->qstage ? 4 : 8;
    rc |= encode_rows(&pl->tmap[KP], d.points, (uint64_t)np, 16);
    if (pl->qstage)
        rc |= encode_rows(&pl->tmap[KQ], pl->qstage, (uint64_t)hp->ncells, sizeof(nln_qcell));
    if (pl->hstage)
        rc |= encode_rows(&pl->tmap[KH], pl->hstage, (uint64_t)hp->ncells, sizeof(nln_hcell));
    if (rc) {
        grav_plan_free(pl);
        return rc;
    }
    d.ngroups = ng;
    d.ncells = hp->ncells;
    d.eps2 = (float)hp->eps2;
    d.qsh = 0.5f * (hp->quad_phi_sign == 0.0f ? 1.0f : hp->quad_phi_sign);
    d.box = hp->box;
    pl->hp.points = nullptr;
    pl->hp.qcells = nullptr;
    pl->hp.hcells = nullptr;
    pl->hp.groups = nullptr;
    pl->hp.pptr = pl->hp.qptr = pl->hp.hptr = nullptr;
    pl->hp.plist = nullptr;
    pl->hp.qlist = pl->hp.hlist = nullptr;
    if (pl->pool) {
        // buffers allocated in stream order on the default stream: complete
        // before other streams use them
        const cudaError_t e = cudaStreamSynchronize(0);
        if (e != cudaSuccess) {
            grav_plan_free(pl);
            return gc::cuda_status(e, "upload: pool allocations");
        }
    }
    *plan_out = pl;
    t_phase[1] = now_s() - t_dev;
    return 0;
}
}  // namespace

extern "C" int grav_groups_upload_CUDA(const grav_problem *hp, const grav_tuning *tuning,
                                       grav_plan **plan_out) {
    return upload_impl(hp, tuning, plan_out, 0);
}

namespace {
template <int KIND>
int launch_kind(grav_plan *pl, const DevProblem &dp, cudaStream_t st) {
    if (dp.nitems[KIND] == 0)
        return 0;
    const int wpb = pl->tune.warps_per_block;
    if (KIND == KP) {
        auto kp = pl->plain ? k_points<true> : k_points<false>;
        int fit = 0;
        GC_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, kp, 256, 0));
        int per_sm = pl->tune.blocks_per_sm > 0 ? std::min(pl->tune.blocks_per_sm, fit) : fit;
        int blocks = std::max(1, per_sm) * pl->nsm;
        blocks = std::min(blocks, (dp.nitems[KP] + 7) / 8);
        kp<<<blocks, 256, 0, st>>>(dp);
        GC_CHECK(cudaGetLastError());
        pl->launches++;
        return 0;
    }
    constexpr bool paired = KIND == KH || (KIND == KQ && GRAV_Q2_PAIRED);
    const size_t smem = (size_t)wpb * (pl->staged ? KindOf<KIND, paired>::warp_bytes
                                                  : KindOf<KIND>::warp_bytes);
    auto kern = pl->staged ? (pl->plain ? k_batch<KIND, true, true> : k_batch<KIND, true, false>)
                           : (pl->plain ? k_batch<KIND, false, true> : k_batch<KIND, false, false>);
    GC_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int fit = 0;
    GC_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, kern, wpb * 32, smem));
    int per_sm = pl->tune.blocks_per_sm > 0 ? std::min(pl->tune.blocks_per_sm, fit) : fit;
    int blocks = std::max(1, per_sm) * pl->nsm;
    blocks = std::min(blocks, (dp.nitems[KIND] + wpb - 1) / wpb);
    kern<<<blocks, wpb * 32, smem, st>>>(pl->tmap[KIND], dp);
    GC_CHECK(cudaGetLastError());
    pl->launches++;
    return 0;
}

// k_ewald_moments: `warps` warps per block, each with two 11 KiB stages,
// blocks_per_sm x SM count blocks (0: as many as fit), at most one warp per
// group; over dp's groups, on stream s.
int launch_moments(grav_plan *pl, const DevProblem &dp, cudaStream_t s, int per_sm, int warps) {
    const int64_t n = dp.ngroups - dp.gbegin;
    if (n <= 0)
        return 0;
    const size_t smem = (size_t)warps * kEwWarpBytes;
    GC_CHECK(cudaFuncSetAttribute(k_ewald_moments, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  4 * kEwWarpBytes));
    if (per_sm <= 0) {
        int fit = 0;
        GC_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, k_ewald_moments, warps * 32,
                                                               smem));
        per_sm = std::max(1, fit);
    }
    DevProblem d = dp;
    d.ewm = pl->ewm;
    const unsigned blocks = (unsigned)std::max<int64_t>(
        1, std::min<int64_t>((n + warps - 1) / warps, (int64_t)per_sm * pl->nsm));
    k_ewald_moments<<<blocks, warps * 32, smem, s>>>(d);
    GC_CHECK(cudaGetLastError());
    pl->launches++;
    return 0;
}

// Placement of the periodic correction moments: ewald_side > 0 runs them on
// a side stream beside the list kernels (k_ewald_side) in that many two-warp
// blocks per SM, sharing the SMs with them; ewald_side = -k runs them
// (k_ewald_moments) on the evaluation's stream between the list kernels and
// the finish pass, with the SMs to themselves, in blocks of k warps (k = 1,
// 2 or 4) as many as fit.  Automatic (0): the side stream with 2 blocks per
// SM while the correction list is short beside the order-4 lists, else the
// evaluation's stream with two-warp blocks.  Measured on one B200: at 256^3
// (MAC 1.5e-6; correction entries 1.2 % of the order-4 interactions) the
// side stream takes 813 ms a step against 825 ms; where the moments take
// half the order-4 kernel's time (128^3, MAC 1e-4) the side stream loses.
int main_moments_warps(const grav_plan *pl) {
    const int k = -pl->tune.ewald_side;
    return (k == 1 || k == 2 || k == 4) ? k : 2;
}

int side_blocks(const grav_plan *pl) {
    if (!pl->dp.ewald || !pl->side || !pl->ewm || pl->tune.ewald_side < 0)
        return 0;
    if (pl->tune.ewald_side > 0)
        return pl->tune.ewald_side;
    return pl->ewald_entries < 0.015 * (double)pl->counts[3] ? 2 : 0;
}

// Fork: k_ewald_moments over dp's groups on the side stream, after the work
// already on st; returns whether it forked (join with side_join).
int side_fork(grav_plan *pl, const DevProblem &dp, cudaStream_t st, bool &forked) {
    forked = false;
    const int per_sm = side_blocks(pl);
    if (per_sm <= 0 || dp.ngroups - dp.gbegin <= 0)
        return 0;
    GC_CHECK(cudaEventRecord(pl->fork, st));
    GC_CHECK(cudaStreamWaitEvent(pl->side, pl->fork, 0));
    DevProblem d = dp;
    d.ewm = pl->ewm;
    const int64_t n = dp.ngroups - dp.gbegin;
    const unsigned blocks =
        (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 1) / 2, (int64_t)per_sm * pl->nsm));
    k_ewald_side<<<blocks, 64, 0, pl->side>>>(d);
    GC_CHECK(cudaGetLastError());
    pl->launches++;
    GC_CHECK(cudaEventRecord(pl->join, pl->side));
    forked = true;
    return 0;
}

int side_join(grav_plan *pl, cudaStream_t st) {
    GC_CHECK(cudaStreamWaitEvent(st, pl->join, 0));
    return 0;
}

// The finish pass, after the correction moments when they did not run on
// the side stream (forked).
int launch_finish(grav_plan *pl, const DevProblem &dp, cudaStream_t st, bool forked) {
    if (dp.ewald && !forked)
        if (int rc = launch_moments(pl, dp, st, 0, main_moments_warps(pl)))
            return rc;
    const int wpb = 2;
    const int64_t n = dp.ngroups - dp.gbegin;
    if (n <= 0)
        return 0;
    k_finish<<<(unsigned)((n + wpb - 1) / wpb), wpb * 32, 0, st>>>(dp);
    GC_CHECK(cudaGetLastError());
    pl->launches++;
    return 0;
}
}  // namespace

extern "C" int grav_groups_eval_CUDA(grav_plan *pl, void *stream) {
    if (!pl)
        return gc::set_status(-1, "grav_groups_eval_CUDA: no plan");
    cudaStream_t st = (cudaStream_t)stream;
    pl->launches = 0;
    auto mark = [&](int k) -> int {
        if (pl->timing)
            GC_CHECK(cudaEventRecord(pl->ev[k], st));
        return 0;
    };
    GC_CHECK(cudaMemsetAsync(pl->dp.counters, 0, 4 * sizeof(int), st));
    if (int rc = mark(0))
        return rc;
    bool forked = false;
    if (int rc = side_fork(pl, pl->dp, st, forked))
        return rc;
    if (int rc = launch_kind<KH>(pl, pl->dp, st))
        return rc;
    if (int rc = mark(1))
        return rc;
    if (int rc = launch_kind<KQ>(pl, pl->dp, st))
        return rc;
    if (int rc = mark(2))
        return rc;
    if (int rc = launch_kind<KP>(pl, pl->dp, st))
        return rc;
    if (int rc = mark(3))
        return rc;
    DevProblem df = pl->dp;
    df.ewm = pl->ewm;
    if (forked)
        if (int rc = side_join(pl, st))
            return rc;
    if (int rc = launch_finish(pl, df, st, forked))
        return rc;
    pl->evaluated = true;
    return mark(4);
}

extern "C" int grav_plan_retune_CUDA(grav_plan *pl, const grav_tuning *tuning) {
    if (!pl || !tuning)
        return gc::set_status(-1, "grav_plan_retune_CUDA: bad arguments");
    const int64_t ng = pl->hp.ngroups;
    grav_tuning t = *tuning;
    if (t.warps_per_block < 1 || t.warps_per_block > 8)
        t.warps_per_block = 8;
    const int64_t tot[3] = {pl->lists_ptr[0].empty() ? 0 : pl->lists_ptr[0][ng],
                            pl->lists_ptr[1].empty() ? 0 : pl->lists_ptr[1][ng],
                            pl->lists_ptr[2].empty() ? 0 : pl->lists_ptr[2][ng]};
    if (t.chunk_p <= 0)
        t.chunk_p = auto_chunk(tot[0], ng, pl->nsm, 128);
    if (t.chunk_q <= 0)
        t.chunk_q = auto_chunk(tot[1], ng, pl->nsm, 64);
    if (t.chunk_h <= 0)
        t.chunk_h = auto_chunk(tot[2], ng, pl->nsm, 32);
    t.ewald_n = pl->tune.ewald_n;  // the correction table is not rebuilt
    pl->tune = t;
    std::vector<Item> items[3];
    std::vector<int64_t> gslot;
    pl->nslots = make_queue(pl, items, gslot);
    // replace the queue's device buffers
    GC_CHECK(cudaDeviceSynchronize());
    auto drop = [&](const void *p) {
        if (!p)
            return;
        auto it = std::find(pl->allocs.begin(), pl->allocs.end(), p);
        if (it != pl->allocs.end()) {
            if (pl->pool)
                cudaFreeAsync(*it, 0);
            else
                cudaFree(*it);
            pl->allocs.erase(it);
        }
    };
    DevProblem &d = pl->dp;
    for (int k = 0; k < 3; k++) drop(d.items[k]);
    drop(d.part);
    drop(d.gslot);
    int rc = 0;
    for (int k = 0; k < 3; k++) {
        Item *it = nullptr;
        rc |= dev_copy(pl, items[k].data(), items[k].size(), &it);
        d.items[k] = it;
        d.nitems[k] = (int)items[k].size();
    }
    float4 *part = nullptr;
    rc |= dev_copy<float4>(pl, nullptr, (size_t)std::max<int64_t>(1, pl->nslots) * 64, &part);
    d.part = part;
    int64_t *gs = nullptr;
    rc |= dev_copy(pl, gslot.data(), gslot.size(), &gs);
    d.gslot = gs;
    if (pl->step)
        step_graph_reset(pl->step);  // a captured step holds the old queue
    return rc;
}

extern "C" int grav_plan_get_tuning(const grav_plan *pl, grav_tuning *out) {
    if (!pl || !out)
        return gc::set_status(-1, "grav_plan_get_tuning: bad arguments");
    *out = pl->tune;
    return 0;
}

extern "C" int grav_plan_set_timing(grav_plan *pl, int on) {
    if (!pl)
        return gc::set_status(-1, "grav_plan_set_timing: no plan");
    if (on && !pl->ev[0])
        for (int k = 0; k < 5; k++) GC_CHECK(cudaEventCreate(&pl->ev[k]));
    pl->timing = on ? 1 : 0;
    return 0;
}

extern "C" int grav_plan_kernel_ms(grav_plan *pl, float ms[4]) {
    if (!pl || !pl->timing)
        return gc::set_status(-1, "grav_plan_kernel_ms: timing is off");
    GC_CHECK(cudaEventSynchronize(pl->ev[4]));
    for (int k = 0; k < 4; k++) GC_CHECK(cudaEventElapsedTime(&ms[k], pl->ev[k], pl->ev[k + 1]));
    return 0;
}

extern "C" int grav_groups_download_CUDA(grav_plan *pl, float *acc_phi) {
    if (!pl || !acc_phi)
        return gc::set_status(-1, "grav_groups_download_CUDA: bad arguments");
    GC_CHECK(cudaMemcpy(acc_phi, pl->dp.out, (size_t)pl->hp.nbodies * sizeof(float4),
                        cudaMemcpyDeviceToHost));
    unsigned h = 0;
    GC_CHECK(cudaMemcpy(&h, pl->dp.err, sizeof(h), cudaMemcpyDeviceToHost));
    if (h) {
        cudaMemset(pl->dp.err, 0, sizeof(unsigned));
        return gc::set_status(-2, "batched kernels: device error word 0x%x", h);
    }
    return 0;
}

extern "C" float *grav_plan_output(grav_plan *pl) {
    return pl ? reinterpret_cast<float *>(pl->dp.out) : nullptr;
}

extern "C" void grav_plan_counts(const grav_plan *pl, int64_t out[4]) {
    for (int k = 0; k < 4; k++) out[k] = pl ? pl->counts[k] : 0;
}

extern "C" int grav_plan_launches(const grav_plan *pl) { return pl ? pl->launches : 0; }

extern "C" void grav_plan_free(grav_plan *pl) {
    if (!pl)
        return;
    if (pl->step)
        step_state_free(pl->step);
    if (pl->adj)
        adjoint_state_free(pl->adj);
    for (void *p : pl->allocs) {
        if (pl->pool)
            cudaFreeAsync(p, 0);  // back to the pool, reserved for the next call
        else
            cudaFree(p);
    }
    for (cudaEvent_t e : pl->ev)
        if (e)
            cudaEventDestroy(e);
    if (pl->side) {
        cudaStreamSynchronize(pl->side);
        cudaStreamDestroy(pl->side);
    }
    if (pl->fork)
        cudaEventDestroy(pl->fork);
    if (pl->join)
        cudaEventDestroy(pl->join);
    delete pl;
}

// step.cuh: the plan's step state adopts a device-built tree's links
int set_tree_adopt(grav_plan *pl, int64_t *cell_first, int32_t *cell_count, int32_t *cell_child,
                   int32_t *cell_nchild, const int32_t *cell_level, cudaMemPool_t pool);

namespace {
// The device build and the plan that adopts it; buffers from the device's
// pool (grav_groups_release_CUDA returns the memory it keeps reserved).
int build_plan(const nln_params *params, const float4 *bodies, int64_t n, double eps2,
               float quad_phi_sign, int ewald, const grav_tuning *tuning, grav_plan **plan) {
    *plan = nullptr;
    cudaMemPool_t pool = nullptr;
    if (int rc = e2e_pool(&pool))
        return rc;
    DevTree T;
    const double t0 = now_s();
    if (int rc = gpu_tree_build(*params, bodies, n, 0, T, pool)) {
        dev_tree_free(T, pool);
        return rc;
    }
    grav_problem hp{};
    hp.nbodies = T.n;
    hp.ncells = T.ncells;
    hp.ngroups = T.ngroups;
    hp.points = reinterpret_cast<const float *>(T.points);
    hp.qcells = T.qcells;
    hp.hcells = T.hcells;
    hp.groups = T.groups_h.data();
    hp.pptr = T.ptr_h[0].data();
    hp.qptr = T.ptr_h[1].data();
    hp.hptr = T.ptr_h[2].data();
    hp.plist = T.list[0];
    hp.qlist = T.list[1];
    hp.hlist = T.list[2];
    hp.eps2 = eps2;
    hp.box = params->box;
    hp.quad_phi_sign = quad_phi_sign;
    hp.ewald = params->box > 0 && ewald;
    hp.cptr = T.ptr_h[3].data();
    hp.clist = T.list[3];
    // the tree's links (for the device refit and the adjoint) stay on the
    // device: the plan's step state adopts them
    int64_t *cfirst = T.cell_first;
    int32_t *ccount = T.cell_count, *cchild = T.cell_child, *cnchild = T.cell_nchild,
            *clevel = T.cell_level;
    T.cell_first = nullptr;
    T.cell_count = T.cell_child = T.cell_nchild = T.cell_level = nullptr;
    grav_plan *pl = nullptr;
    if (int rc = upload_impl(&hp, tuning, &pl, 0, &T)) {
        for (void *q : {(void *)cfirst, (void *)ccount, (void *)cchild, (void *)cnchild,
                        (void *)clevel})
            cudaFreeAsync(q, 0);
        return rc;  // upload_impl took the tree's other buffers over and released them
    }
    const int rc_links = set_tree_adopt(pl, cfirst, ccount, cchild, cnchild, clevel, pool);
    cudaFreeAsync(clevel, 0);
    if (rc_links) {
        grav_plan_free(pl);
        return rc_links;
    }
    t_build = now_s() - t0;
    for (int k = 0; k < 6; k++) t_build_phase[k] = T.seconds[k];
    *plan = pl;
    return 0;
}

// out[order[i]] = in[i]: results from tree order back to the input order.
__global__ void k_unorder(const float4 *__restrict__ in, const int64_t *__restrict__ order,
                          int64_t n, float4 *out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const int64_t j = order[i];
        if (j >= 0 && j < n)
            out[j] = in[i];
    }
}
}  // namespace

extern "C" int grav_plan_build_CUDA(const nln_params *params, const float *bodies, int64_t n,
                                    double eps2, float quad_phi_sign, int ewald,
                                    const grav_tuning *tuning, grav_plan **plan) {
    if (!params || !bodies || !plan || n <= 0)
        return gc::set_status(-1, "grav_plan_build_CUDA: bad arguments");
    *plan = nullptr;
    if (((uintptr_t)bodies & 15u) != 0)
        return gc::set_status(-1, "grav_plan_build_CUDA: bodies must be 16-byte aligned");
    return build_plan(params, reinterpret_cast<const float4 *>(bodies), n, eps2, quad_phi_sign,
                      ewald, tuning, plan);
}

extern "C" int grav_build_eval_CUDA(const nln_params *params, const float *bodies, int64_t n,
                                    double eps2, float quad_phi_sign, int ewald,
                                    float *acc_phi) {
    if (!params || !bodies || !acc_phi || n <= 0)
        return gc::set_status(-1, "grav_build_eval_CUDA: bad arguments");
    const double t_start = now_s();
    cudaMemPool_t pool = nullptr;
    if (int rc = e2e_pool(&pool))
        return rc;
    float4 *dev = nullptr, *out = nullptr;
    const size_t bytes = (size_t)n * sizeof(float4);
    GC_CHECK(cudaMallocFromPoolAsync((void **)&dev, bytes, pool, 0));
    cudaError_t e = cudaMallocFromPoolAsync((void **)&out, bytes, pool, 0);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dev, bodies, bytes, cudaMemcpyHostToDevice, 0);
    if (e != cudaSuccess) {
        cudaFreeAsync(dev, 0);
        if (out)
            cudaFreeAsync(out, 0);
        return gc::cuda_status(e, "grav_build_eval_CUDA: bodies");
    }
    const double t_h2d = now_s();
    grav_plan *pl = nullptr;
    int rc = build_plan(params, dev, n, eps2, quad_phi_sign, ewald, nullptr, &pl);
    const double t_built = now_s();
    if (!rc)
        rc = grav_groups_eval_CUDA(pl, nullptr);
    if (!rc) {
        k_unorder<<<(unsigned)((n + 255) / 256), 256>>>(pl->dp.out, pl->order, n, out);
        e = cudaGetLastError();
        if (e == cudaSuccess)
            e = cudaMemcpy(acc_phi, out, bytes, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess)
            rc = gc::cuda_status(e, "grav_build_eval_CUDA: results");
    }
    const double t_eval = now_s();
    if (!rc) {
        unsigned h = 0;
        e = cudaMemcpy(&h, pl->dp.err, sizeof(h), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess)
            rc = gc::cuda_status(e, "grav_build_eval_CUDA: error word");
        else if (h)
            rc = gc::set_status(-2, "grav_build_eval_CUDA: device error word 0x%x", h);
    }
    if (pl)
        grav_plan_free(pl);
    cudaFreeAsync(dev, 0);
    cudaFreeAsync(out, 0);
    cudaStreamSynchronize(0);
    t_phase_be[0] = t_h2d - t_start;
    t_phase_be[1] = t_built - t_h2d;
    t_phase_be[2] = t_eval - t_built;
    t_phase_be[3] = now_s() - t_eval;
    return rc;
}

extern "C" void grav_build_eval_phases(double seconds[4]) {
    for (int k = 0; k < 4; k++) seconds[k] = t_phase_be[k];
}

extern "C" const int64_t *grav_plan_order(const grav_plan *pl) { return pl ? pl->order : nullptr; }

extern "C" void grav_plan_build_phases(double seconds[7]) {
    for (int k = 0; k < 6; k++) seconds[k] = t_build_phase[k];
    seconds[6] = t_build;
}

extern "C" int grav_plan_problem(const grav_plan *pl, grav_problem *out) {
    if (!pl || !out)
        return gc::set_status(-1, "grav_plan_problem: bad arguments");
    *out = pl->hp;
    const DevProblem &d = pl->dp;
    out->points = reinterpret_cast<const float *>(d.points);
    out->qcells = d.qcells;
    out->hcells = d.hcells;
    out->groups = d.groups;
    out->plist = d.list[0];
    out->qlist = d.list[1];
    out->hlist = d.list[2];
    out->clist = d.clist;
    auto host = [&](int k) { return pl->lists_ptr[k].empty() ? nullptr : pl->lists_ptr[k].data(); };
    out->pptr = host(0);
    out->qptr = host(1);
    out->hptr = host(2);
    out->cptr = host(3);
    for (int k = 0; k < 4; k++) {
        out->zptr[k] = nullptr;
        out->zlist[k] = nullptr;
    }
    return 0;
}

namespace {
// Group ranges of the pipelined end-to-end call: one per 2 GiB of list
// words copied (packed words where a kind is run-packed), at most 16, the
// first one split further; GRAV_E2E_CHUNKS overrides the count.
int e2e_chunks(const grav_problem *hp) {
    if (const char *e = getenv("GRAV_E2E_CHUNKS"))
        return std::max(1, std::min(64, atoi(e)));
    const int64_t ng = hp->ngroups;
    const int64_t *plain[4] = {hp->pptr, hp->qptr, hp->hptr,
                               hp->box > 0 && hp->ewald ? hp->cptr : nullptr};
    int64_t words = 0;
    for (int k = 0; k < 4; k++) {
        if (!plain[k])
            continue;
        words += (hp->zlist[k] && hp->zptr[k]) ? hp->zptr[k][ng] : plain[k][ng];
    }
    return (int)std::max<int64_t>(1, std::min<int64_t>(16, (words * 4 + (2ll << 30) - 1) >> 31));
}

// Copy group range c's slice of every list on `cs`, then make `st` wait for it.
int copy_range(grav_plan *pl, const grav_problem *hp, size_t c, cudaStream_t cs, cudaStream_t st,
               cudaEvent_t ev) {
    const int64_t g0 = pl->chunk_group[c], g1 = pl->chunk_group[c + 1];
    const DevProblem &d = pl->dp;
    const int64_t *ptr[4] = {hp->pptr, hp->qptr, hp->hptr, d.clist ? hp->cptr : nullptr};
    const uint32_t *src[4] = {hp->plist, hp->qlist, hp->hlist, hp->clist};
    const uint32_t *dst[4] = {d.list[0], d.list[1], d.list[2], d.clist};
    for (int k = 0; k < 4; k++) {
        if (pl->zdev[k]) {  // run-packed: copy the words, k_unpack fills dst
            ptr[k] = hp->zptr[k];
            src[k] = hp->zlist[k];
            dst[k] = pl->zdev[k];
        }
        if (!ptr[k] || !dst[k] || ptr[k][g1] <= ptr[k][g0])
            continue;
        GC_CHECK(cudaMemcpyAsync(const_cast<uint32_t *>(dst[k]) + ptr[k][g0], src[k] + ptr[k][g0],
                                 (size_t)(ptr[k][g1] - ptr[k][g0]) * sizeof(uint32_t),
                                 cudaMemcpyHostToDevice, cs));
    }
    GC_CHECK(cudaEventRecord(ev, cs));
    GC_CHECK(cudaStreamWaitEvent(st, ev, 0));
    return 0;
}

// Evaluate group range c: its work items, then its groups' finish pass.
int eval_range(grav_plan *pl, size_t c, cudaStream_t st) {
    DevProblem dp = pl->dp;
    for (int k = 0; k < 3; k++) {
        const int b = pl->chunk_item[k][c], e = pl->chunk_item[k][c + 1];
        dp.items[k] = pl->dp.items[k] ? pl->dp.items[k] + b : nullptr;
        dp.nitems[k] = e - b;
    }
    dp.counters = pl->dp.counters + 4 * c;
    dp.gbegin = pl->chunk_group[c];
    dp.ngroups = pl->chunk_group[c + 1];
    for (int k = 0; k < 4; k++) {
        if (!pl->zdev[k])
            continue;
        uint32_t *dst = const_cast<uint32_t *>(k < 3 ? pl->dp.list[k] : pl->dp.clist);
        const int64_t n = dp.ngroups - dp.gbegin;
        const unsigned blocks = (unsigned)std::max<int64_t>(
            1, std::min<int64_t>((n + 7) / 8, (int64_t)pl->nsm * 16));
        k_unpack<<<blocks, 256, 0, st>>>(pl->zdev[k], pl->zptr_dev[k], pl->lptr_dev[k], dp.gbegin,
                                         dp.ngroups, dst, pl->dp.err);
        GC_CHECK(cudaGetLastError());
        pl->launches++;
    }
    bool forked = false;
    int rc = side_fork(pl, dp, st, forked);
    if (!rc)
        rc = launch_kind<KH>(pl, dp, st);
    if (!rc)
        rc = launch_kind<KQ>(pl, dp, st);
    if (!rc)
        rc = launch_kind<KP>(pl, dp, st);
    dp.ewm = pl->ewm;
    if (!rc && forked)
        rc = side_join(pl, st);
    if (!rc)
        rc = launch_finish(pl, dp, st, forked);
    return rc;
}
}  // namespace

// The end-to-end call: upload the tables, then copy the lists range by range
// on a copy stream while the kernels evaluate the ranges already copied, and
// download.  Lists in page-locked host memory overlap best; pageable lists
// still overlap each copy with the previous range's kernels.
extern "C" int grav_groups_CUDA(const grav_problem *hp, float *acc_phi) {
    if (!hp || hp->ngroups <= 0 || !hp->pptr || !acc_phi)
        return gc::set_status(-1, "grav_groups_CUDA: incomplete problem");
    grav_plan *pl = nullptr;
    if (hp->lists_in_host) {
        if (int rc = grav_groups_upload_CUDA(hp, nullptr, &pl))
            return rc;
        double t0 = now_s();
        int rc = grav_groups_eval_CUDA(pl, nullptr);
        const cudaError_t e = rc ? cudaSuccess : cudaDeviceSynchronize();
        if (e != cudaSuccess)
            rc = gc::cuda_status(e, "grav_groups_CUDA: evaluation");
        t_phase[2] = now_s() - t0;
        t0 = now_s();
        if (!rc)
            rc = grav_groups_download_CUDA(pl, acc_phi);
        t_phase[3] = now_s() - t0;
        t0 = now_s();
        grav_plan_free(pl);
        t_phase[4] = now_s() - t0;
        return rc;
    }
    if (int rc = upload_impl(hp, nullptr, &pl, e2e_chunks(hp)))
        return rc;
    const size_t nc = pl->chunk_group.size() - 1;
    double t0 = now_s();
    auto chk = [](cudaError_t e, const char *what) {
        return e == cudaSuccess ? 0 : gc::cuda_status(e, what);
    };
    // one copy stream and one compute stream (ranges alternating over two
    // compute streams measured no faster: their kernels compete for the SMs)
    cudaStream_t cs = nullptr, st = nullptr;
    std::vector<cudaEvent_t> ev(nc, nullptr);
    int rc = 0;
    cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    for (size_t c = 0; c < nc && e == cudaSuccess; c++)
        e = cudaEventCreateWithFlags(&ev[c], cudaEventDisableTiming);
    rc = chk(e, "grav_groups_CUDA: streams");
    if (!rc)
        rc = chk(cudaMemsetAsync(pl->dp.counters, 0, 4 * nc * sizeof(int), st),
                 "grav_groups_CUDA: queue heads");
    pl->launches = 0;
    for (size_t c = 0; c < nc && !rc; c++) {
        rc = copy_range(pl, hp, c, cs, st, ev[c]);
        if (!rc)
            rc = eval_range(pl, c, st);
    }
    if (!rc)
        rc = chk(cudaStreamSynchronize(st), "grav_groups_CUDA: evaluation");
    t_phase[2] = now_s() - t0;
    t0 = now_s();
    if (!rc)
        rc = grav_groups_download_CUDA(pl, acc_phi);
    t_phase[3] = now_s() - t0;
    t0 = now_s();
    if (cs)
        cudaStreamSynchronize(cs);
    if (st)
        cudaStreamSynchronize(st);
    for (cudaEvent_t x : ev)
        if (x)
            cudaEventDestroy(x);
    if (cs)
        cudaStreamDestroy(cs);
    if (st)
        cudaStreamDestroy(st);
    grav_plan_free(pl);
    t_phase[4] = now_s() - t0;
    return rc;
}

extern "C" void grav_groups_release_CUDA(void) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    if (dev >= 0 && dev < kMaxPoolDevices && g_pool[dev]) {
        cudaDeviceSynchronize();
        cudaMemPoolTrimTo(g_pool[dev], 0);
    }
}

extern "C" void grav_groups_CUDA_phases(double seconds[5]) {
    for (int k = 0; k < 5; k++) seconds[k] = t_phase[k];
}

// ------------------------------------------------------------ no-allocation evaluation
//
// grav_groups_eval_dev_CUDA runs the batched kernels above on a problem that
// is already on the device, with every byte of scratch taken from this one
// file-scope array: queue counters and the error word, one work item per
// (group, list kind), a checked copy of the groups, the slot offsets and
// the per-item partial sums.  Its address is looked up once per device.
static __device__ __align__(256) unsigned char g_dev_scratch[GRAV_DEV_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;

struct DevScratch {
    int *counters;      // 4 queue heads: must be 0 when the kernels start
    unsigned *err;      // device error word: must be 0 when the kernels start
    Item *items[3];
    nln_group *groups;  // checked copy of the caller's groups
    int64_t *gslot;
    float4 *part;
};

size_t round256(size_t b) { return (b + 255) / 256 * 256; }

// Scratch bytes for ng groups with nk list kinds.
size_t dev_scratch_bytes(int64_t ng, int nk) {
    return 256 + 3 * round256((size_t)ng * sizeof(Item)) + round256((size_t)ng * sizeof(nln_group)) +
           round256((size_t)(ng + 1) * sizeof(int64_t)) + (size_t)nk * ng * 64 * sizeof(float4);
}

// Once per device, with that device current: the scratch's address, the
// device's SM count and the shared-memory attribute of the two row-gather
// kernels this entry launches (point lists run in k_points, which needs none).
int dev_scratch_base(void **out, int *nsm) {
    static std::mutex mu;
    static void *base[kMaxDevices] = {};
    static int sms[kMaxDevices] = {};
    int dev = 0;
    GC_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        return gc::set_status(-1, "grav_groups_eval_dev_CUDA: device %d beyond %d", dev, kMaxDevices);
    std::lock_guard<std::mutex> lk(mu);
    if (!base[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_dev_scratch);
        if (e != cudaSuccess)
            return gc::cuda_status(e, "grav_groups_eval_dev_CUDA: cudaGetSymbolAddress of the scratch");
        if (!p)
            return gc::set_status(-1, "grav_groups_eval_dev_CUDA: the scratch has no device address");
        int n = 0;
        e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess)
            return gc::cuda_status(e, "grav_groups_eval_dev_CUDA: SM count");
        if (n <= 0)
            return gc::set_status(-1, "grav_groups_eval_dev_CUDA: device %d reports no SMs", dev);
        GC_CHECK(cudaFuncSetAttribute(k_batch<KQ, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      8 * KindOf<KQ>::warp_bytes));
        GC_CHECK(cudaFuncSetAttribute(k_batch<KH, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      8 * KindOf<KH>::warp_bytes));
        sms[dev] = n;
        base[dev] = p;
    }
    *out = base[dev];
    *nsm = sms[dev];
    return 0;
}

// One thread per group: check the group and its list offsets, copy it, and
// write its work items (slot nk*g + kind rank) and slot offset.  A group
// that fails the checks flags GC_DEV_BAD_INDEX and becomes one sink (body
// 0) with empty lists, so no kernel leaves the tables.
__global__ void k_dev_setup(const nln_group *__restrict__ groups, const int64_t *p0,
                            const int64_t *p1, const int64_t *p2, int64_t ng, int64_t nbodies,
                            int nk, DevScratch S) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g == 0)
        S.gslot[ng] = (int64_t)nk * ng;
    if (g >= ng)
        return;
    nln_group G = groups[g];
    const int64_t *ptr[3] = {p0, p1, p2};
    bool ok = G.count >= 1 && G.count <= 32 && G.first >= 0 && G.first + G.count <= nbodies;
    for (int k = 0; k < 3; k++)
        if (ptr[k] && (ptr[k][g] < 0 || ptr[k][g + 1] < ptr[k][g]))
            ok = false;
    if (!ok) {
        atomicOr(S.err, GC_DEV_BAD_INDEX);
        G.first = 0;
        G.count = 1;
    }
    S.groups[g] = G;
    int rank = 0;
    for (int k = 0; k < 3; k++) {
        if (!ptr[k])
            continue;
        const int64_t b = ok ? ptr[k][g] : 0, e = ok ? ptr[k][g + 1] : 0;
        S.items[k][g] = Item{(int32_t)g, (int32_t)((int64_t)nk * g + rank), b, e};
        rank++;
    }
    S.gslot[g] = (int64_t)nk * g;
}

}  // namespace

extern "C" int grav_groups_eval_dev_CUDA(const grav_problem *dp, float *acc_phi, void *stream) {
    if (!dp || !acc_phi || dp->nbodies <= 0 || dp->ngroups <= 0 || !dp->points || !dp->groups ||
        !dp->pptr || !dp->plist)
        return gc::set_status(-1, "grav_groups_eval_dev_CUDA: incomplete problem");
    if (dp->box > 0 && dp->ewald)
        return gc::set_status(-1, "grav_groups_eval_dev_CUDA: no Ewald correction here (its table "
                                  "is a per-plan allocation); use grav_groups_upload_CUDA");
    if (dp->nbodies + dp->ncells >= (int64_t)NLN_IDX_MASK)
        return gc::set_status(-1, "grav_groups_eval_dev_CUDA: point table exceeds 27-bit indices");
    if ((dp->qptr && (!dp->qlist || !dp->qcells)) || (dp->hptr && (!dp->hlist || !dp->hcells)))
        return gc::set_status(-1, "grav_groups_eval_dev_CUDA: a cell list without its table");
    auto misaligned = [](const void *p) { return ((uintptr_t)p & 15u) != 0; };
    if (misaligned(dp->points) || misaligned(dp->qcells) || misaligned(dp->hcells) ||
        misaligned(acc_phi))
        return gc::set_status(-1, "grav_groups_eval_dev_CUDA: tables and output must be "
                                  "16-byte aligned");
    const int64_t ng = dp->ngroups, np = dp->nbodies + dp->ncells;
    const int nk = 1 + (dp->qptr ? 1 : 0) + (dp->hptr ? 1 : 0);
    const size_t need = dev_scratch_bytes(ng, nk);
    if (need > (size_t)GRAV_DEV_SCRATCH_BYTES) {
        int64_t fit = 0;
        while (dev_scratch_bytes(fit + 1, nk) <= (size_t)GRAV_DEV_SCRATCH_BYTES) fit += 1;
        return gc::set_status(-1, "grav_groups_eval_dev_CUDA: %lld groups need %zu bytes of "
                                  "scratch; the static scratch holds %zu (at most %lld groups with "
                                  "%d list kinds)",
                              (long long)ng, need, (size_t)GRAV_DEV_SCRATCH_BYTES, (long long)fit, nk);
    }
    void *basev = nullptr;
    int nsm = 0;
    if (int rc = dev_scratch_base(&basev, &nsm))
        return rc;
    unsigned char *base = static_cast<unsigned char *>(basev);
    DevScratch S{};
    size_t off = 0;
    S.counters = reinterpret_cast<int *>(base);
    S.err = reinterpret_cast<unsigned *>(base + 4 * sizeof(int));
    off = 256;
    for (int k = 0; k < 3; k++) {
        S.items[k] = reinterpret_cast<Item *>(base + off);
        off += round256((size_t)ng * sizeof(Item));
    }
    S.groups = reinterpret_cast<nln_group *>(base + off);
    off += round256((size_t)ng * sizeof(nln_group));
    S.gslot = reinterpret_cast<int64_t *>(base + off);
    off += round256((size_t)(ng + 1) * sizeof(int64_t));
    S.part = reinterpret_cast<float4 *>(base + off);

    // a plan on the stack: device pointers only, nothing owned
    grav_plan pl;
    pl.nsm = nsm;
    pl.tune = default_tuning();
    DevProblem &d = pl.dp;
    d.points = reinterpret_cast<const float4 *>(dp->points);
    d.qcells = dp->qptr ? dp->qcells : nullptr;
    d.hcells = dp->hptr ? dp->hcells : nullptr;
    d.groups = S.groups;
    const int64_t *ptrs[3] = {dp->pptr, dp->qptr, dp->hptr};
    const uint32_t *lists[3] = {dp->plist, dp->qlist, dp->hlist};
    for (int k = 0; k < 3; k++) {
        d.list[k] = ptrs[k] ? lists[k] : nullptr;
        d.items[k] = ptrs[k] ? S.items[k] : nullptr;
        d.nitems[k] = ptrs[k] ? (int)ng : 0;
    }
    d.ntab[0] = np;
    d.ntab[1] = d.ntab[2] = dp->ncells;
    d.counters = S.counters;
    d.part = S.part;
    d.gslot = S.gslot;
    d.out = reinterpret_cast<float4 *>(acc_phi);
    d.ngroups = ng;
    d.ncells = dp->ncells;
    d.eps2 = (float)dp->eps2;
    d.qsh = 0.5f * (dp->quad_phi_sign == 0.0f ? 1.0f : dp->quad_phi_sign);
    d.box = dp->box;
    d.err = S.err;
    d.cptr = nullptr;
    d.clist = nullptr;
    d.ewald = 0;
    memset(pl.tmap, 0, sizeof(pl.tmap));
    int rc = encode_rows(&pl.tmap[KP], d.points, (uint64_t)np, 16);
    if (!rc && d.qcells)
        rc = encode_rows(&pl.tmap[KQ], d.qcells, (uint64_t)dp->ncells, sizeof(nln_qcell));
    if (!rc && d.hcells)
        rc = encode_rows(&pl.tmap[KH], d.hcells, (uint64_t)dp->ncells, sizeof(nln_hcell));
    if (rc)
        return rc;

    cudaStream_t st = (cudaStream_t)stream;
    GC_CHECK(cudaMemsetAsync(base, 0, 256, st));  // queue counters and error word
    // From here on work is queued on the shared scratch: every return waits
    // for the stream first, so that no call leaves kernels behind that could
    // still write the scratch when the next call starts.
    auto finish = [&](int status) {
        const cudaError_t e = cudaStreamSynchronize(st);
        if (status)
            return status;
        return e == cudaSuccess ? 0 : gc::cuda_status(e, "grav_groups_eval_dev_CUDA: evaluation");
    };
    k_dev_setup<<<(unsigned)((ng + 255) / 256), 256, 0, st>>>(dp->groups, dp->pptr, dp->qptr,
                                                               dp->hptr, ng, dp->nbodies, nk, S);
    if (cudaError_t e = cudaGetLastError(); e != cudaSuccess)
        return finish(gc::cuda_status(e, "grav_groups_eval_dev_CUDA: setup launch"));
    if ((rc = launch_kind<KH>(&pl, pl.dp, st)) || (rc = launch_kind<KQ>(&pl, pl.dp, st)) ||
        (rc = launch_kind<KP>(&pl, pl.dp, st)))
        return finish(rc);
    k_finish<<<(unsigned)((ng + 7) / 8), 256, 0, st>>>(pl.dp);
    if (cudaError_t e = cudaGetLastError(); e != cudaSuccess)
        return finish(gc::cuda_status(e, "grav_groups_eval_dev_CUDA: finish launch"));
    unsigned h = 0;
    if (cudaError_t e = cudaMemcpyAsync(&h, S.err, sizeof(h), cudaMemcpyDeviceToHost, st);
        e != cudaSuccess)
        return finish(gc::cuda_status(e, "grav_groups_eval_dev_CUDA: reading the error word"));
    if (int r = finish(0))
        return r;
    if (h)
        return gc::set_status(-2, "grav_groups_eval_dev_CUDA: device error word 0x%x", h);
    return 0;
}

#include "step.cuh"
#include "adjoint.cuh"
