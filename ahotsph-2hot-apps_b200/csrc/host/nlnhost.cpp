// nlnhost.cpp -- host tree build, FP64 moments, AREL critical radii, group MAC
// walk and list packing (the producer side of the gravcuda.h boundary).
//
// Algorithms restated from the reference (file:line in lanl/ahotsph-2hot-apps):
//   moments and their normalisation   nln/cofm.c:96-231, 398-420, 486-562
//   AREL critical radii               nln/cofm.c:276-565, rcrit_poly/rtnewt 577-624
//   MAC acceptance order m -> q -> h  nln/mac.c:1785-1805 (DLRcritMAC)
//   leaf expansion to bodies          nln/mac.c:1817-1832
//   completeness invariant            nln/mac.c:734-735
//   image offsets                     nln/mac.c:91-111
// The oct-tree itself comes from the absent 2hot libtree; this is a fresh
// implementation (Morton keys, level-synchronous split).  The walk is a
// group walk: every sink group (a tree cell with <= group_max bodies) keeps
// one list, and the MAC distance is reduced by the group radius so that
// every sink of the group satisfies the reference's per-sink test.
#include "nlnhost.h"

#include <omp.h>

#include "tree_math.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <parallel/algorithm>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

struct Cell {
    int64_t first;
    int32_t count;
    int32_t child;   // first child cell, -1 for a leaf
    int32_t nchild;
    int32_t level;
    double gc[3];    // geometric cube centre
    double side;     // cube side
    double cen[3];   // expansion centre: centre of mass
    double mass, bmax, B2, B4, B6;
    double rc_m, rc_q, rc_h;
};

inline uint64_t spread3(uint32_t v) {
    uint64_t x = v & 0x1fffff;
    x = (x | x << 32) & 0x1f00000000ffffULL;
    x = (x | x << 16) & 0x1f0000ff0000ffULL;
    x = (x | x << 8) & 0x100f00f00f00f00fULL;
    x = (x | x << 4) & 0x10c30c30c30c30c3ULL;
    x = (x | x << 2) & 0x1249249249249249ULL;
    return x;
}

constexpr int KEY_LEVELS = 21;

}  // namespace

// A list array left uninitialised at allocation (its pages are committed as
// the walk writes them) and released explicitly.
struct ListBuf {
    std::unique_ptr<uint32_t[]> p;
    size_t n = 0;
    void alloc(size_t count) {
        p.reset(count ? new uint32_t[count] : nullptr);
        n = count;
    }
    void release() {
        p.reset();
        n = 0;
    }
    uint32_t *data() { return p.get(); }
    const uint32_t *data() const { return p.get(); }
    size_t size() const { return n; }
    uint32_t operator[](size_t i) const { return p[i]; }
};

struct nln_tree {
    nln_params p{};
    int64_t n = 0;
    double origin[3] = {0, 0, 0};
    double side = 0;
    std::vector<int64_t> order;
    std::vector<float> spos;   // xyz in tree order
    std::vector<float> smass;
    std::vector<Cell> cells;
    std::vector<float> points;  // float4
    std::vector<nln_qcell> qc;
    std::vector<nln_hcell> hc;
    std::vector<nln_group> groups;
    
    std::vector<int64_t> lptr[4];
    ListBuf plist;
    ListBuf qlist, hlist;
    ListBuf clist;  // periodic correction list
    std::vector<int64_t> zptr[4];  // run-packed lists (nln_tree_pack)
    ListBuf zlist[4];
    std::vector<nln_wcell> wcells;  // what the walk reads of each cell (built by nln_tree_walk)
    std::vector<int64_t> aptr[3];
    std::vector<float> adata[3];
    int64_t counts[4] = {0, 0, 0, 0};
    int merged = 0;  // a batch of trees (nln_tree_merge): several roots, no re-walk
};

extern "C" const char *nln_last_error(void) { return g_err.c_str(); }

static int nthreads_of(const nln_params &p) {
    return p.nthreads > 0 ? p.nthreads : omp_get_max_threads();
}

// ---------------------------------------------------------------- build
static void build_cells(nln_tree *t, const std::vector<uint64_t> &keys) {
    const int leaf_max = t->p.leaf_max;
    Cell root{};
    root.first = 0;
    root.count = (int32_t)t->n;
    root.child = -1;
    root.level = 0;
    for (int d = 0; d < 3; d++) root.gc[d] = t->origin[d] + 0.5 * t->side;
    root.side = t->side;
    t->cells.push_back(root);
    std::vector<int32_t> frontier{0};
    while (!frontier.empty()) {
        const int64_t nf = (int64_t)frontier.size();
        std::vector<int32_t> nkids(nf, 0);
        std::vector<int64_t> bounds(nf * 9, 0);
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t f = 0; f < nf; f++) {
            const Cell &c = t->cells[frontier[f]];
            if (c.count <= leaf_max || c.level >= KEY_LEVELS)
                continue;
            const int shift = 3 * (KEY_LEVELS - 1 - c.level);
            int64_t lo = c.first, hi = c.first + c.count;
            bounds[f * 9] = lo;
            int nk = 0;
            for (int o = 0; o < 8; o++) {
                // first key whose octant digit exceeds o
                int64_t a = lo, b = hi;
                while (a < b) {
                    int64_t mid = (a + b) / 2;
                    if ((int)((keys[mid] >> shift) & 7) <= o)
                        a = mid + 1;
                    else
                        b = mid;
                }
                bounds[f * 9 + o + 1] = a;
                if (a > lo)
                    nk++;
                lo = a;
            }
            nkids[f] = nk;
        }
        std::vector<int64_t> off(nf + 1, 0);
        for (int64_t f = 0; f < nf; f++) off[f + 1] = off[f] + nkids[f];
        const int64_t base = (int64_t)t->cells.size();
        t->cells.resize(base + off[nf]);
        std::vector<int32_t> next(off[nf]);
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t f = 0; f < nf; f++) {
            if (!nkids[f])
                continue;
            Cell &c = t->cells[frontier[f]];
            c.child = (int32_t)(base + off[f]);
            c.nchild = nkids[f];
            int k = 0;
            for (int o = 0; o < 8; o++) {
                int64_t lo = bounds[f * 9 + o], hi = bounds[f * 9 + o + 1];
                if (hi <= lo)
                    continue;
                Cell d{};
                d.first = lo;
                d.count = (int32_t)(hi - lo);
                d.child = -1;
                d.level = c.level + 1;
                d.side = 0.5 * c.side;
                d.gc[0] = c.gc[0] + ((o >> 2) & 1 ? 0.25 : -0.25) * c.side;
                d.gc[1] = c.gc[1] + ((o >> 1) & 1 ? 0.25 : -0.25) * c.side;
                d.gc[2] = c.gc[2] + ((o >> 0) & 1 ? 0.25 : -0.25) * c.side;
                t->cells[base + off[f] + k] = d;
                next[off[f] + k] = (int32_t)(base + off[f] + k);
                k++;
            }
        }
        frontier.swap(next);
    }
}

// The canonical order of every per-cell FP64 sum over a cell's bodies, which
// the GPU tree builder reproduces exactly: bodies in blocks of 64 summed in
// order, those partials in blocks of 64 summed in order, then those summed
// in order.  term(k, acc) adds body k's K terms into acc.
constexpr int kSumBlock = 64;

template <int K, typename Term>
static void canon_sum(int32_t count, Term term, double out[K]) {
    for (int q = 0; q < K; q++) out[q] = 0.0;
    const int32_t nb0 = (count + kSumBlock - 1) / kSumBlock;
    const int32_t nb1 = (nb0 + kSumBlock - 1) / kSumBlock;
    for (int32_t b1 = 0; b1 < nb1; b1++) {
        double p1[K] = {};
        for (int32_t b0 = b1 * kSumBlock; b0 < std::min(nb0, (b1 + 1) * kSumBlock); b0++) {
            double p0[K] = {};
            for (int32_t k = b0 * kSumBlock; k < std::min(count, (b0 + 1) * kSumBlock); k++)
                term(k, p0);
            for (int q = 0; q < K; q++) p1[q] += p0[q];
        }
        for (int q = 0; q < K; q++) out[q] += p1[q];
    }
}

// FP64 moments about the centre of mass, directly from the bodies of each
// cell (canon_sum order), then the traceless R^-l normalisation of
// nln/cofm.c:398-420,486-562.
static void compute_moments(nln_tree *t) {
    const int64_t nc = (int64_t)t->cells.size();
    t->qc.assign(nc, nln_qcell{});
    t->hc.assign(nc, nln_hcell{});
    t->points.resize((size_t)(t->n + nc) * 4);
    for (int64_t i = 0; i < t->n; i++) {
        for (int d = 0; d < 3; d++) t->points[4 * i + d] = t->spos[3 * i + d];
        t->points[4 * i + 3] = t->smass[i];
    }
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t ci = 0; ci < nc; ci++) {
        Cell &c = t->cells[ci];
        const float *P = t->spos.data() + 3 * c.first;
        const float *M = t->smass.data() + c.first;
        double s1[4];
        canon_sum<4>(c.count, [&](int32_t k, double *a) { nln_mass_terms(P + 3 * k, M[k], c.gc, a); },
                     s1);
        const double m = s1[0];
        for (int d = 0; d < 3; d++) c.cen[d] = c.gc[d] + (m > 0 ? s1[1 + d] / m : 0.0);
        c.mass = m;
        // raw moments about cen (layout of nln_moment_terms) and the largest r^2
        double mo[NLN_NMOM];
        double bmax2 = 0;
        canon_sum<NLN_NMOM>(c.count, [&](int32_t k, double *a) {
            bmax2 = std::max(bmax2, nln_moment_terms(P + 3 * k, M[k], c.cen, a));
        }, mo);
        c.bmax = std::sqrt(bmax2);
        c.B2 = mo[31];
        c.B4 = mo[32];
        c.B6 = mo[33];
        nln_cell_tables(c.cen, m, c.bmax, mo, &t->points[4 * (t->n + ci)], &t->qc[ci], &t->hc[ci]);
    }
}

// The MAC parameters of a tree (nln_cell_rcrit, nln_walk_group).
static nln_mac mac_of(const nln_tree *t) {
    nln_mac P;
    P.tol = t->p.tol;
    P.rel_tol = t->p.rel_tol;
    P.rel_tol0 = t->p.rel_tol0;
    P.ptol_boost = t->p.ptol_boost;
    P.bmax0 = 0.5 * t->side;  // mac->bmax0 = r0, cofm.c:66
    P.p2cut = t->p.p2cut;
    P.p4cut = t->p.p4cut;
    P.box = t->p.box;
    P.ewald_theta = t->p.ewald_theta;
    return P;
}

// AREL critical radii of every cell (nln_cell_rcrit).
static void compute_rcrit(nln_tree *t) {
    const nln_mac P = mac_of(t);
    const int64_t nc = (int64_t)t->cells.size();
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t ci = 0; ci < nc; ci++) {
        Cell &c = t->cells[ci];
        double rc[3];
        nln_cell_rcrit(P, c.count, c.mass, c.bmax, c.B2, c.B4, c.B6, rc);
        c.rc_m = rc[0];
        c.rc_q = rc[1];
        c.rc_h = rc[2];
    }
}

// Sink groups: the largest cells with <= group_max bodies, then consecutive
// sibling cells merged while the merged group still holds <= group_max
// bodies (siblings are adjacent in key order, so a merged group is still one
// contiguous run of sinks inside its parent's cube).
static void collect_groups(nln_tree *t) {
    const int gmax = t->p.group_max;
    struct Run {
        int64_t first;
        int32_t count;
    };
    std::vector<Run> runs;
    std::vector<int32_t> stack{0};
    while (!stack.empty()) {
        int32_t ci = stack.back();
        stack.pop_back();
        const Cell &c = t->cells[ci];
        if (c.count <= gmax || c.child < 0) {
            runs.push_back(Run{c.first, c.count});
            continue;
        }
        // children of c that are small enough: merge adjacent ones greedily
        std::vector<Run> merged;
        std::vector<int32_t> big;
        for (int k = 0; k < c.nchild; k++) {
            const Cell &d = t->cells[c.child + k];
            if (d.count > gmax && d.child >= 0) {
                big.push_back(c.child + k);
                continue;
            }
            if (!merged.empty() && merged.back().first + merged.back().count == d.first &&
                merged.back().count + d.count <= gmax)
                merged.back().count += d.count;
            else
                merged.push_back(Run{d.first, d.count});
        }
        runs.insert(runs.end(), merged.begin(), merged.end());
        for (auto it = big.rbegin(); it != big.rend(); ++it) stack.push_back(*it);
    }
    std::sort(runs.begin(), runs.end(), [](const Run &a, const Run &b) { return a.first < b.first; });
    // a leaf that cannot split further (coincident bodies at the deepest key
    // level) can hold more than gmax bodies: its run becomes consecutive
    // groups of gmax, the last one the remainder
    std::vector<Run> pieces;
    pieces.reserve(runs.size());
    for (const Run &r : runs)
        for (int32_t k = 0; k < r.count; k += gmax)
            pieces.push_back(Run{r.first + k, std::min<int32_t>(gmax, r.count - k)});
    runs.swap(pieces);
    t->groups.resize(runs.size());
#pragma omp parallel for schedule(static)
    for (size_t g = 0; g < runs.size(); g++) {
        nln_group &G = t->groups[g];
        const float *P = t->spos.data() + 3 * runs[g].first;
        const float *M = t->smass.data() + runs[g].first;
        double m = 0, s[3] = {0, 0, 0};
        for (int32_t k = 0; k < runs[g].count; k++) {
            m += M[k];
            for (int d = 0; d < 3; d++) s[d] += M[k] * (double)P[3 * k + d];
        }
        double r2max = 0;
        for (int d = 0; d < 3; d++) G.cen[d] = m > 0 ? s[d] / m : (double)P[d];
        for (int32_t k = 0; k < runs[g].count; k++) {
            double r2 = 0;
            for (int d = 0; d < 3; d++) {
                double x = (double)P[3 * k + d] - G.cen[d];
                r2 += x * x;
            }
            r2max = std::max(r2max, r2);
        }
        G.first = runs[g].first;
        G.count = runs[g].count;
        G.radius = (float)(std::sqrt(r2max) * (1.0 + 1e-6));
    }
}

extern "C" nln_tree *nln_tree_build(const float *pos, int stride, const float *mass, int mstride,
                                    int64_t n, const nln_params *p) {
    if (!pos || !mass || !p || n <= 0 || stride < 3 || mstride < 1) {
        g_err = "nln_tree_build: bad arguments";
        return nullptr;
    }
    if (p->leaf_max < 1 || p->leaf_max > 65535 || p->group_max < 1 || p->group_max > 64 ||
        p->tol <= 0.0 || p->p2cut < 0 || p->p4cut < 0) {
        g_err = "nln_tree_build: bad parameters (leaf_max 1..65535, group_max 1..64, tol > 0)";
        return nullptr;
    }
    if (n + 1 >= (int64_t)NLN_IDX_MASK) {
        g_err = "nln_tree_build: too many bodies for 27-bit list indices";
        return nullptr;
    }
    nln_tree *t = new nln_tree();
    t->p = *p;
    t->n = n;
    const int nth = nthreads_of(*p);
    omp_set_num_threads(nth);
    // bounding cube
    if (p->box > 0) {
        for (int64_t i = 0; i < n; i++)
            for (int d = 0; d < 3; d++) {
                float x = pos[i * stride + d];
                if (!(x >= 0.0f && (double)x < p->box)) {
                    g_err = "nln_tree_build: periodic body outside [0, box)";
                    delete t;
                    return nullptr;
                }
            }
        t->side = p->box;
    } else {
        double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int64_t i = 0; i < n; i++)
            for (int d = 0; d < 3; d++) {
                double x = pos[i * stride + d];
                if (!std::isfinite(x)) {
                    g_err = "nln_tree_build: non-finite position";
                    delete t;
                    return nullptr;
                }
                lo[d] = std::min(lo[d], x);
                hi[d] = std::max(hi[d], x);
            }
        double ext = 0;
        for (int d = 0; d < 3; d++) ext = std::max(ext, hi[d] - lo[d]);
        ext = ext > 0 ? ext * (1.0 + 1e-5) : 1.0;
        for (int d = 0; d < 3; d++) t->origin[d] = 0.5 * (lo[d] + hi[d]) - 0.5 * ext;
        t->side = ext;
    }
    // keys + sort
    struct KI {
        uint64_t k;
        int64_t i;
    };
    std::vector<KI> ki(n);
    const double scale = (double)(1u << KEY_LEVELS) / t->side;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
        uint32_t c[3];
        for (int d = 0; d < 3; d++) {
            double u = ((double)pos[i * stride + d] - t->origin[d]) * scale;
            int64_t v = (int64_t)std::floor(u);
            v = std::min<int64_t>(std::max<int64_t>(v, 0), (1 << KEY_LEVELS) - 1);
            c[d] = (uint32_t)v;
        }
        ki[i].k = spread3(c[0]) << 2 | spread3(c[1]) << 1 | spread3(c[2]);
        ki[i].i = i;
    }
    __gnu_parallel::sort(ki.begin(), ki.end(), [](const KI &a, const KI &b) {
        return a.k < b.k || (a.k == b.k && a.i < b.i);
    });
    std::vector<uint64_t> keys(n);
    t->order.resize(n);
    t->spos.resize(3 * n);
    t->smass.resize(n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
        keys[i] = ki[i].k;
        int64_t j = ki[i].i;
        t->order[i] = j;
        for (int d = 0; d < 3; d++) t->spos[3 * i + d] = pos[j * stride + d];
        t->smass[i] = mass[j * mstride];
    }
    build_cells(t, keys);
    compute_moments(t);
    compute_rcrit(t);
    collect_groups(t);
    return t;
}

extern "C" void nln_tree_free(nln_tree *t) { delete t; }

// ---------------------------------------------------------------- walk
namespace {

struct GroupLists {
    std::vector<uint32_t> p;   // point-table record | image << 27
    std::vector<uint32_t> q, h;
    std::vector<uint32_t> c;   // periodic correction: point-table record | image << 27
    int64_t nb = 0, nm = 0;
};

// Host emitter of nln_walk_group: the group's lists as vectors.
struct HostEmit {
    GroupLists &L;
    void p(uint32_t e, bool body) {
        L.p.push_back(e);
        if (body)
            L.nb++;
        else
            L.nm++;
    }
    void q(uint32_t e) { L.q.push_back(e); }
    void h(uint32_t e) { L.h.push_back(e); }
    void c(uint32_t e) { L.c.push_back(e); }
};

}  // namespace

// One group's walk (nln_walk_group over the tree's walk records).
static void walk_group(const nln_tree *t, const nln_group &G, GroupLists &L,
                       std::vector<int32_t> &stack) {
    HostEmit em{L};
    const int rc = nln_walk_group(t->wcells.data(), t->spos.data(), t->n, G, mac_of(t),
                                  stack.data(), (int)stack.size(), em);
    if (rc) {
        std::fprintf(stderr, "nln_tree_walk: group at %lld: %s\n", (long long)G.first,
                     rc == -1 ? "does not cover every body exactly once" : "walk stack overflow");
        std::abort();
    }
}


static void emit_aosoa(nln_tree *t, const std::vector<GroupLists> &GL) {
    const int64_t ng = (int64_t)t->groups.size();
    const int SZ[3] = {4, 13, 29};
    const double box = t->p.box;
    for (int kind = 0; kind < 3; kind++) {
        std::vector<int64_t> &ptr = t->aptr[kind];
        ptr.assign(ng + 1, 0);
        for (int64_t g = 0; g < ng; g++) {
            int64_t nrec = 0;
            nrec = (int64_t)(kind == 0 ? GL[g].p.size()
                                       : (kind == 1 ? GL[g].q.size() : GL[g].h.size()));
            ptr[g + 1] = ptr[g] + (nrec + 7) / 8;
        }
        t->adata[kind].assign((size_t)ptr[ng] * SZ[kind] * 8, 0.0f);
    }
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t g = 0; g < ng; g++) {
        // M list: bodies and monopole cells, [m, x, y, z]
        {
            float *f = t->adata[0].data() + (size_t)t->aptr[0][g] * 4 * 8;
            int64_t r = 0;
            for (const uint32_t e : GL[g].p) {
                const uint32_t sc = e >> NLN_IDX_BITS;
                int sh[3] = {(int)sc / 9 - 1, (int)(sc / 3) % 3 - 1, (int)sc % 3 - 1};
                const float *pt = &t->points[4 * (size_t)(e & NLN_IDX_MASK)];
                float *blk = f + (r / 8) * 4 * 8;
                int l = (int)(r % 8);
                blk[0 * 8 + l] = pt[3];
                for (int d = 0; d < 3; d++)
                    blk[(1 + d) * 8 + l] = (float)((double)pt[d] + sh[d] * box);
                r++;
            }
        }
        for (int kind = 1; kind < 3; kind++) {
            const std::vector<uint32_t> &lst = kind == 1 ? GL[g].q : GL[g].h;
            const int sz = SZ[kind];
            float *f = t->adata[kind].data() + (size_t)t->aptr[kind][g] * sz * 8;
            for (size_t r = 0; r < lst.size(); r++) {
                uint32_t ci = lst[r] & NLN_IDX_MASK, sc = lst[r] >> NLN_IDX_BITS;
                int sh[3] = {(int)sc / 9 - 1, (int)(sc / 3) % 3 - 1, (int)sc % 3 - 1};
                const nln_hcell &h = t->hc[ci];
                float *blk = f + (r / 8) * sz * 8;
                int l = (int)(r % 8);
                blk[0 * 8 + l] = h.mass;
                for (int d = 0; d < 3; d++) blk[(1 + d) * 8 + l] = (float)(h.cen[d] + sh[d] * box);
                blk[4 * 8 + l] = h.R;
                for (int k = 0; k < 5; k++) blk[(8 + k) * 8 + l] = h.q2[k];
                if (kind == 2) {
                    for (int k = 0; k < 7; k++) blk[(13 + k) * 8 + l] = h.q3[k];
                    for (int k = 0; k < 9; k++) blk[(20 + k) * 8 + l] = h.q4[k];
                }
            }
        }
    }
}

extern "C" int nln_tree_walk(nln_tree *t) {
    if (!t)
        return -1;
    if (t->merged) {
        g_err = "nln_tree_walk: a merged batch keeps its members' lists";
        return -1;
    }
    omp_set_num_threads(nthreads_of(t->p));
    const int64_t ng = (int64_t)t->groups.size();
    const int64_t ncell = (int64_t)t->cells.size();
    t->wcells.resize(ncell);
#pragma omp parallel for schedule(static)
    for (int64_t ci = 0; ci < ncell; ci++) {
        const Cell &c = t->cells[ci];
        nln_wcell &w = t->wcells[ci];
        for (int d = 0; d < 3; d++) w.cen[d] = c.cen[d];
        w.bmax = c.bmax;
        w.rc[0] = c.rc_m;
        w.rc[1] = c.rc_q;
        w.rc[2] = c.rc_h;
        w.first = c.first;
        w.count = c.count;
        w.child = c.child;
        w.nchild = c.nchild;
        w.pad = 0;
    }
    // Groups are walked in chunks.  Each chunk's lists are packed into one
    // exact-size segment per kind, and its per-group vectors are reused by
    // the next chunk, so the host holds about one copy of the lists (plus
    // one segment while they are joined), not per-group vectors and the
    // final arrays at once.  The AoSoA emitter needs every group's vectors:
    // then there is a single chunk.
    const int64_t chunk = t->p.emit_aosoa ? std::max<int64_t>(ng, 1) : 16384;
    std::vector<GroupLists> GL((size_t)std::min<int64_t>(ng, chunk));
    struct Segment {
        ListBuf part[4];
    };
    std::vector<Segment> segs;
    for (int k = 0; k < 4; k++) t->lptr[k].assign(ng + 1, 0);
    int64_t cnt[4] = {0, 0, 0, 0};
    for (int64_t c0 = 0; c0 < ng; c0 += chunk) {
        const int64_t c1 = std::min(ng, c0 + chunk);
#pragma omp parallel
        {
            std::vector<int32_t> stack(NLN_WALK_STACK);
#pragma omp for schedule(dynamic, 8)
            for (int64_t g = c0; g < c1; g++) {
                GroupLists &L = GL[g - c0];
                L.p.clear();
                L.q.clear();
                L.h.clear();
                L.c.clear();
                L.nb = L.nm = 0;
                walk_group(t, t->groups[g], L, stack);
            }
        }
        for (int64_t g = c0; g < c1; g++) {
            const GroupLists &L = GL[g - c0];
            t->lptr[0][g + 1] = t->lptr[0][g] + (int64_t)L.p.size();
            t->lptr[1][g + 1] = t->lptr[1][g] + (int64_t)L.q.size();
            t->lptr[2][g + 1] = t->lptr[2][g] + (int64_t)L.h.size();
            t->lptr[3][g + 1] = t->lptr[3][g] + (int64_t)L.c.size();
            const int64_t gc = t->groups[g].count;
            cnt[0] += gc * L.nb;
            cnt[1] += gc * L.nm;
            cnt[2] += gc * (int64_t)L.q.size();
            cnt[3] += gc * (int64_t)L.h.size();
        }
        Segment S;
        for (int k = 0; k < 4; k++) S.part[k].alloc((size_t)(t->lptr[k][c1] - t->lptr[k][c0]));
#pragma omp parallel for schedule(static)
        for (int64_t g = c0; g < c1; g++) {
            const GroupLists &L = GL[g - c0];
            const std::vector<uint32_t> *src[4] = {&L.p, &L.q, &L.h, &L.c};
            for (int k = 0; k < 4; k++)
                std::copy(src[k]->begin(), src[k]->end(),
                          S.part[k].data() + (t->lptr[k][g] - t->lptr[k][c0]));
        }
        segs.push_back(std::move(S));
    }
    std::memcpy(t->counts, cnt, sizeof(cnt));
    for (int k = 0; k < 4; k++) {  // packed forms of earlier lists are stale
        t->zptr[k].clear();
        t->zlist[k].release();
    }
    ListBuf *dst[4] = {&t->plist, &t->qlist, &t->hlist, &t->clist};
    for (int k = 0; k < 4; k++) {
        dst[k]->alloc((size_t)t->lptr[k][ng]);
        size_t off = 0;
        for (Segment &S : segs) {
            const size_t n = S.part[k].size();
            uint32_t *d = dst[k]->data() + off;
            const uint32_t *sp = S.part[k].data();
#pragma omp parallel for schedule(static)
            for (int64_t b = 0; b < (int64_t)((n + 65535) / 65536); b++) {
                const size_t lo = (size_t)b * 65536, hi = std::min(n, lo + 65536);
                std::memcpy(d + lo, sp + lo, (hi - lo) * sizeof(uint32_t));
            }
            off += n;
            S.part[k].release();
        }
    }
    if (t->p.emit_aosoa)
        emit_aosoa(t, GL);
    return 0;
}

// ---------------------------------------------------------------- accessors
extern "C" int64_t nln_nbodies(const nln_tree *t) { return t->n; }
extern "C" int64_t nln_ncells(const nln_tree *t) { return (int64_t)t->cells.size(); }
extern "C" int64_t nln_ngroups(const nln_tree *t) { return (int64_t)t->groups.size(); }
extern "C" const int64_t *nln_order(const nln_tree *t) { return t->order.data(); }
extern "C" const float *nln_points(const nln_tree *t) { return t->points.data(); }
extern "C" const nln_qcell *nln_qcells(const nln_tree *t) { return t->qc.data(); }
extern "C" const nln_hcell *nln_hcells(const nln_tree *t) { return t->hc.data(); }
extern "C" const nln_group *nln_groups(const nln_tree *t) { return t->groups.data(); }
extern "C" const float *nln_sorted_pos(const nln_tree *t) { return t->spos.data(); }

extern "C" const int64_t *nln_list_ptr(const nln_tree *t, int kind) {
    return (kind >= 0 && kind < 4 && !t->lptr[kind].empty()) ? t->lptr[kind].data() : nullptr;
}
extern "C" const void *nln_list_data(const nln_tree *t, int kind) {
    if (kind == 0)
        return t->plist.data();
    if (kind == 1)
        return t->qlist.data();
    if (kind == 2)
        return t->hlist.data();
    if (kind == 3)
        return t->clist.data();
    return nullptr;
}
extern "C" int64_t nln_list_len(const nln_tree *t, int kind) {
    if (kind == 0)
        return (int64_t)t->plist.size();
    if (kind == 1)
        return (int64_t)t->qlist.size();
    if (kind == 2)
        return (int64_t)t->hlist.size();
    if (kind == 3)
        return (int64_t)t->clist.size();
    return -1;
}
extern "C" void nln_counts(const nln_tree *t, int64_t out[4]) {
    std::memcpy(out, t->counts, sizeof(t->counts));
}
extern "C" const int64_t *nln_aosoa_ptr(const nln_tree *t, int kind) {
    return (kind >= 0 && kind < 3 && !t->aptr[kind].empty()) ? t->aptr[kind].data() : nullptr;
}
extern "C" const float *nln_aosoa_data(const nln_tree *t, int kind) {
    return (kind >= 0 && kind < 3 && !t->adata[kind].empty()) ? t->adata[kind].data() : nullptr;
}

// ---------------------------------------------------------------- run packing
// Words of one group's packed list; with out != nullptr they are written.
// A run shorter than 3 entries stays as plain entries (a run word saves
// nothing there).
static int64_t pack_group(const uint32_t *e, int64_t n, uint32_t *out) {
    int64_t w = 0, i = 0;
    while (i < n) {
        const uint32_t v = e[i];
        int64_t j = i + 1;
        while (j < n && e[j] == v + (uint32_t)(j - i) && (e[j] >> NLN_IDX_BITS) == (v >> NLN_IDX_BITS) &&
               (uint64_t)(j - i) < (uint64_t)NLN_IDX_MASK)
            j++;
        const int64_t len = j - i;
        if (len >= 3) {
            if (out) {
                out[w] = v;
                out[w + 1] = (NLN_RUN_CODE << NLN_IDX_BITS) | (uint32_t)(len - 1);
            }
            w += 2;
        } else {
            for (int64_t k = 0; k < len; k++)
                if (out)
                    out[w + k] = e[i + k];
            w += len;
        }
        i = j;
    }
    return w;
}

extern "C" int nln_tree_pack(nln_tree *t) {
    const int64_t ng = (int64_t)t->groups.size();
    if (ng == 0 || t->lptr[0].empty()) {
        g_err = "nln_tree_pack: no lists (walk the tree first)";
        return -1;
    }
    const ListBuf *src[4] = {&t->plist, &t->qlist, &t->hlist, &t->clist};
    for (int k = 0; k < 4; k++) {
        t->zptr[k].clear();
        t->zlist[k].release();
        if (t->lptr[k].empty())
            continue;
        const int64_t *ptr = t->lptr[k].data();
        const uint32_t *e = src[k]->data();
        std::vector<int64_t> &z = t->zptr[k];
        z.assign(ng + 1, 0);
#pragma omp parallel for schedule(dynamic, 1024)
        for (int64_t g = 0; g < ng; g++) z[g + 1] = pack_group(e + ptr[g], ptr[g + 1] - ptr[g], nullptr);
        for (int64_t g = 0; g < ng; g++) z[g + 1] += z[g];
        t->zlist[k].alloc((size_t)z[ng]);
        uint32_t *out = t->zlist[k].data();
#pragma omp parallel for schedule(dynamic, 1024)
        for (int64_t g = 0; g < ng; g++) pack_group(e + ptr[g], ptr[g + 1] - ptr[g], out + z[g]);
    }
    return 0;
}

extern "C" const int64_t *nln_packed_ptr(const nln_tree *t, int kind) {
    return (kind >= 0 && kind < 4 && !t->zptr[kind].empty()) ? t->zptr[kind].data() : nullptr;
}
extern "C" const uint32_t *nln_packed_data(const nln_tree *t, int kind) {
    return (kind >= 0 && kind < 4) ? t->zlist[kind].data() : nullptr;
}
extern "C" int64_t nln_packed_len(const nln_tree *t, int kind) {
    return (kind >= 0 && kind < 4 && !t->zptr[kind].empty()) ? (int64_t)t->zlist[kind].size() : -1;
}

// Reference AoSoA blocks (nln/mac.c:117-153) for a subset of groups, packed
// from the index lists: kind 0 = M (bodies and monopole cells, MSZ 4), 1 = Q
// (QSZ 13), 2 = H (HSZ 29).  With data == NULL only blk_ptr (ngsel + 1
// entries) is filled; the return value is the total block count.
extern "C" int64_t nln_aosoa_subset(const nln_tree *t, const int64_t *gids, int64_t ngsel,
                                    int kind, int64_t *blk_ptr, float *data) {
    if (!t || kind < 0 || kind > 2 || t->lptr[kind].empty())
        return -1;
    static const int SZ[3] = {4, 13, 29};
    const int sz = SZ[kind];
    const ListBuf &lst = kind == 0 ? t->plist : (kind == 1 ? t->qlist : t->hlist);
    const int64_t *ptr = t->lptr[kind].data();
    blk_ptr[0] = 0;
    for (int64_t s = 0; s < ngsel; s++) {
        const int64_t g = gids[s];
        blk_ptr[s + 1] = blk_ptr[s] + (ptr[g + 1] - ptr[g] + 7) / 8;
    }
    if (!data)
        return blk_ptr[ngsel];
    const double box = t->p.box;
#pragma omp parallel for schedule(dynamic, 8)
    for (int64_t s = 0; s < ngsel; s++) {
        const int64_t g = gids[s];
        float *f = data + (size_t)blk_ptr[s] * sz * 8;
        std::fill(f, f + (size_t)(blk_ptr[s + 1] - blk_ptr[s]) * sz * 8, 0.0f);
        for (int64_t r = 0; r < ptr[g + 1] - ptr[g]; r++) {
            const uint32_t e = lst[ptr[g] + r];
            const uint32_t idx = e & NLN_IDX_MASK, sc = e >> NLN_IDX_BITS;
            const int sh[3] = {(int)sc / 9 - 1, (int)(sc / 3) % 3 - 1, (int)sc % 3 - 1};
            float *blk = f + (r / 8) * sz * 8;
            const int l = (int)(r % 8);
            if (kind == 0) {
                const float *pt = &t->points[4 * (size_t)idx];
                blk[l] = pt[3];
                for (int d = 0; d < 3; d++)
                    blk[(1 + d) * 8 + l] = (float)((double)pt[d] + sh[d] * box);
            } else {
                const nln_hcell &h = t->hc[idx];
                blk[l] = h.mass;
                for (int d = 0; d < 3; d++) blk[(1 + d) * 8 + l] = (float)(h.cen[d] + sh[d] * box);
                blk[4 * 8 + l] = h.R;
                for (int k = 0; k < 5; k++) blk[(8 + k) * 8 + l] = h.q2[k];
                if (kind == 2) {
                    for (int k = 0; k < 7; k++) blk[(13 + k) * 8 + l] = h.q3[k];
                    for (int k = 0; k < 9; k++) blk[(20 + k) * 8 + l] = h.q4[k];
                }
            }
        }
    }
    return blk_ptr[ngsel];
}

// Body range of every cell (tree order): bodies [first[c], first[c] + count[c]).
extern "C" void nln_cell_ranges(const nln_tree *t, int64_t *first, int32_t *count) {
    for (size_t c = 0; c < t->cells.size(); c++) {
        first[c] = t->cells[c].first;
        count[c] = t->cells[c].count;
    }
}

extern "C" nln_tree *nln_tree_merge(nln_tree *const *trees, int ntrees) {
    if (!trees || ntrees < 1) {
        g_err = "nln_tree_merge: no trees";
        return nullptr;
    }
    int64_t nb = 0, nc = 0, ng = 0, nl[3] = {0, 0, 0};
    std::vector<int64_t> bo(ntrees), co(ntrees), go(ntrees), lo[3];
    for (int k = 0; k < 3; k++) lo[k].resize(ntrees);
    for (int i = 0; i < ntrees; i++) {
        const nln_tree *t = trees[i];
        if (!t || t->p.box > 0 || t->lptr[0].empty() || t->merged) {
            g_err = "nln_tree_merge: every member must be an isolated, walked tree";
            return nullptr;
        }
        bo[i] = nb;
        co[i] = nc;
        go[i] = ng;
        for (int k = 0; k < 3; k++) {
            lo[k][i] = nl[k];
            nl[k] += t->lptr[k].back();
        }
        nb += t->n;
        nc += (int64_t)t->cells.size();
        ng += (int64_t)t->groups.size();
    }
    if (nb + nc >= (int64_t)NLN_IDX_MASK) {
        g_err = "nln_tree_merge: bodies plus cells exceed 27-bit list indices";
        return nullptr;
    }
    nln_tree *m = new nln_tree();
    m->p = trees[0]->p;
    m->merged = 1;
    m->n = nb;
    m->order.resize(nb);
    m->spos.resize(3 * nb);
    m->smass.resize(nb);
    m->cells.resize(nc);
    m->points.resize(4 * (nb + nc));
    m->qc.resize(nc);
    m->hc.resize(nc);
    m->groups.resize(ng);
    for (int k = 0; k < 4; k++) m->lptr[k].assign(ng + 1, 0);
    m->plist.alloc(nl[0]);
    m->qlist.alloc(nl[1]);
    m->hlist.alloc(nl[2]);
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < ntrees; i++) {
        const nln_tree *t = trees[i];
        const int64_t b0 = bo[i], c0 = co[i], g0 = go[i];
        for (int64_t j = 0; j < t->n; j++) {
            m->order[b0 + j] = b0 + t->order[j];
            for (int d = 0; d < 3; d++) m->spos[3 * (b0 + j) + d] = t->spos[3 * j + d];
            m->smass[b0 + j] = t->smass[j];
            for (int d = 0; d < 4; d++) m->points[4 * (b0 + j) + d] = t->points[4 * j + d];
        }
        const int64_t tc = (int64_t)t->cells.size();
        for (int64_t c = 0; c < tc; c++) {
            Cell cc = t->cells[c];
            cc.first += b0;
            if (cc.child >= 0)
                cc.child += (int32_t)c0;
            m->cells[c0 + c] = cc;
            for (int d = 0; d < 4; d++)
                m->points[4 * (nb + c0 + c) + d] = t->points[4 * (t->n + c) + d];
            m->qc[c0 + c] = t->qc[c];
            m->hc[c0 + c] = t->hc[c];
        }
        for (size_t g = 0; g < t->groups.size(); g++) {
            nln_group G = t->groups[g];
            G.first += b0;
            m->groups[g0 + g] = G;
            for (int k = 0; k < 3; k++) m->lptr[k][g0 + g + 1] = lo[k][i] + t->lptr[k][g + 1];
        }
        const uint32_t tn = (uint32_t)t->n;
        for (int64_t e = 0; e < t->lptr[0].back(); e++) {
            const uint32_t v = t->plist[e], idx = v & NLN_IDX_MASK, hi = v & ~NLN_IDX_MASK;
            const uint32_t r = idx < tn ? (uint32_t)b0 + idx : (uint32_t)(nb + c0) + (idx - tn);
            m->plist.data()[lo[0][i] + e] = r | hi;
        }
        const ListBuf *src[2] = {&t->qlist, &t->hlist};
        ListBuf *dst[2] = {&m->qlist, &m->hlist};
        for (int k = 0; k < 2; k++)
            for (int64_t e = 0; e < t->lptr[k + 1].back(); e++) {
                const uint32_t v = (*src[k])[e];
                dst[k]->data()[lo[k + 1][i] + e] = ((v & NLN_IDX_MASK) + (uint32_t)c0) |
                                                    (v & ~NLN_IDX_MASK);
            }
    }
    for (int i = 0; i < ntrees; i++)
        for (int k = 0; k < 4; k++) m->counts[k] += trees[i]->counts[k];
    return m;
}

extern "C" void nln_cell_links(const nln_tree *t, int32_t *child, int32_t *nchild,
                               int32_t *level) {
    for (size_t c = 0; c < t->cells.size(); c++) {
        child[c] = t->cells[c].child;
        nchild[c] = t->cells[c].nchild;
        level[c] = t->cells[c].level;
    }
}

extern "C" int nln_tree_refit(nln_tree *t, const float *pos) {
    if (!t || !pos)
        return -1;
    omp_set_num_threads(nthreads_of(t->p));
    std::memcpy(t->spos.data(), pos, sizeof(float) * 3 * (size_t)t->n);
    compute_moments(t);
    return 0;
}
