// step.cuh -- the time step on the device: refit of the cell tables after
// bodies move, the KDK integrator, and one step (evaluate, integrate,
// refit) captured once into a CUDA graph and replayed.
//
// Included once, at the end of batch.cu: it works on the plan's tables.
//
// Refit.  The host builds the tree and the lists; between rebuilds the
// bodies move and every cell record is recomputed from them, deepest level
// first.  A leaf sums over its bodies in FP64 (centre of mass, then the raw
// central moments S_n[alpha] = sum m x^alpha, |alpha| = 2..4, and bmax); a
// parent combines its children with the parallel-axis shift
//     S'[alpha] = sum_child sum_{beta <= alpha} C(alpha, beta) S_child[beta] d^(alpha-beta),
// d = child centre - parent centre (S_0 = m, S_1 = 0 about each centre), as
// nln/cofm.c mpole_add (770-964) shifts moments; a parent's bmax is the
// bound max(|d| + bmax_child).  The tables then take the traceless moments
// normalised by R = bmax exactly as the host does (nln/cofm.c:398-420,
// 486-562), so kernels see R^l q_l, which does not depend on R.  The lists,
// the critical radii and the sink groups (whose centres are only the
// re-centring origin) stay as built.
//
// Integrator.  nln/integrate.c:16-59 (Integrate) per body: the velocity
// synchronised to the positions' time, vc = v + (tpos - tvel) a, gives
// ke += m vc.vc and pe += m phi; then v += dtv a and x += dt v.  KE = ke/2,
// PE = pe/2 (G = 1 here; the caller scales).
#pragma once

namespace {

constexpr int kRaw = 36;  // per cell: m, X[3], S2[6], S3[10], S4[15], bmax

__device__ __forceinline__ int mi3(int ax, int ay, int az) {
    const int n = ax + ay + az;
    return n * (n + 1) * (n + 2) / 6 + (ay + az) * (ay + az + 1) / 2 + az;
}
__device__ __forceinline__ double binom(int n, int k) {
    return (k == 0 || k == n) ? 1.0 : (k == 1 || k == n - 1) ? (double)n : (n == 4 ? 6.0 : 3.0);
}

// raw[kRaw] layout: [0] m, [1..3] X, then S_n at 4 + (mi3 - 4) for |alpha| = 2..4
// (mi3 of order 2 starts at 4, so S[alpha] sits at raw[mi3(alpha)]), [35] bmax.
__global__ void k_refit_level(const float4 *__restrict__ pts, const int64_t *__restrict__ cfirst,
                              const int32_t *__restrict__ ccount, const int32_t *__restrict__ cchild,
                              const int32_t *__restrict__ cnchild, const int32_t *__restrict__ order,
                              int64_t lo, int64_t hi, double *__restrict__ raw) {
    const int64_t i = lo + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= hi)
        return;
    const int32_t c = order[i];
    double R[kRaw];
#pragma unroll
    for (int q = 0; q < kRaw; q++) R[q] = 0.0;
    if (cchild[c] < 0) {
        const int64_t f = cfirst[c];
        const int32_t n = ccount[c];
        if (n > 0) {
            const float4 p0 = pts[f];
            double m = 0, s0 = 0, s1 = 0, s2 = 0;
            for (int32_t k = 0; k < n; k++) {
                const float4 p = pts[f + k];
                m += p.w;
                s0 += p.w * ((double)p.x - p0.x);
                s1 += p.w * ((double)p.y - p0.y);
                s2 += p.w * ((double)p.z - p0.z);
            }
            const double X0 = p0.x + (m > 0 ? s0 / m : 0.0), X1 = p0.y + (m > 0 ? s1 / m : 0.0),
                         X2 = p0.z + (m > 0 ? s2 / m : 0.0);
            R[0] = m;
            R[1] = X0;
            R[2] = X1;
            R[3] = X2;
            double b2 = 0;
            for (int32_t k = 0; k < n; k++) {
                const float4 p = pts[f + k];
                const double d[3] = {(double)p.x - X0, (double)p.y - X1, (double)p.z - X2};
                b2 = fmax(b2, d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                double px[5], py[5], pz[5];
                px[0] = p.w;  // the mass rides on the x powers
                py[0] = 1.0;
                pz[0] = 1.0;
#pragma unroll
                for (int e = 1; e < 5; e++) {
                    px[e] = px[e - 1] * d[0];
                    py[e] = py[e - 1] * d[1];
                    pz[e] = pz[e - 1] * d[2];
                }
#pragma unroll
                for (int a0 = 0; a0 <= 4; a0++)
#pragma unroll
                    for (int a1 = 0; a1 <= 4; a1++)
#pragma unroll
                        for (int a2 = 0; a2 <= 4; a2++)
                            if (a0 + a1 + a2 >= 2 && a0 + a1 + a2 <= 4)
                                R[mi3(a0, a1, a2)] += px[a0] * py[a1] * pz[a2];
            }
            R[35] = sqrt(b2);
        }
    } else {
        const int32_t c0 = cchild[c], nc = cnchild[c];
        double m = 0, s[3] = {0, 0, 0};
        for (int32_t k = 0; k < nc; k++) {
            const double *Q = raw + (size_t)(c0 + k) * kRaw;
            m += Q[0];
            for (int d = 0; d < 3; d++) s[d] += Q[0] * Q[1 + d];
        }
        const double X[3] = {m > 0 ? s[0] / m : 0.0, m > 0 ? s[1] / m : 0.0,
                             m > 0 ? s[2] / m : 0.0};
        R[0] = m;
        R[1] = X[0];
        R[2] = X[1];
        R[3] = X[2];
        double bmax = 0;
        for (int32_t k = 0; k < nc; k++) {
            const double *Q = raw + (size_t)(c0 + k) * kRaw;
            if (Q[0] == 0.0)
                continue;
            const double d[3] = {Q[1] - X[0], Q[2] - X[1], Q[3] - X[2]};
            bmax = fmax(bmax, sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) + Q[35]);
            double px[5], py[5], pz[5];
            px[0] = py[0] = pz[0] = 1.0;
#pragma unroll
            for (int e = 1; e < 5; e++) {
                px[e] = px[e - 1] * d[0];
                py[e] = py[e - 1] * d[1];
                pz[e] = pz[e - 1] * d[2];
            }
            // S'[alpha] += sum_{beta <= alpha, |beta| != 1} C(alpha, beta) S[beta] d^(alpha - beta)
#pragma unroll
            for (int a0 = 0; a0 <= 4; a0++)
#pragma unroll
                for (int a1 = 0; a1 <= 4; a1++)
#pragma unroll
                    for (int a2 = 0; a2 <= 4; a2++) {
                        if (a0 + a1 + a2 < 2 || a0 + a1 + a2 > 4)
                            continue;
                        double acc = Q[0] * px[a0] * py[a1] * pz[a2];  // beta = 0
#pragma unroll
                        for (int b0 = 0; b0 <= a0; b0++)
#pragma unroll
                            for (int b1 = 0; b1 <= a1; b1++)
#pragma unroll
                                for (int b2 = 0; b2 <= a2; b2++) {
                                    const int nb = b0 + b1 + b2;
                                    if (nb < 2)
                                        continue;
                                    acc += binom(a0, b0) * binom(a1, b1) * binom(a2, b2) *
                                           Q[mi3(b0, b1, b2)] * px[a0 - b0] * py[a1 - b1] *
                                           pz[a2 - b2];
                                }
                        R[mi3(a0, a1, a2)] += acc;
                    }
        }
        R[35] = bmax;
    }
    double *out = raw + (size_t)c * kRaw;
#pragma unroll
    for (int q = 0; q < kRaw; q++) out[q] = R[q];
}

// Raw moments -> table records (the host's traceless forms, nlnhost.cpp
// compute_moments, after nln/cofm.c:398-420,507-558).
__global__ void k_refit_tables(const double *__restrict__ raw, int64_t ncells, int64_t nbodies,
                               float4 *__restrict__ pts, nln_qcell *__restrict__ qc,
                               nln_hcell *__restrict__ hc) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells)
        return;
    const double *Q = raw + (size_t)c * kRaw;
    const double m = Q[0], bmax = Q[35];
    auto S = [&](int a0, int a1, int a2) { return Q[mi3(a0, a1, a2)]; };
    const double x2 = S(2, 0, 0), xy = S(1, 1, 0), xz = S(1, 0, 1), y2 = S(0, 2, 0),
                 yz = S(0, 1, 1), z2 = S(0, 0, 2);
    const double x3 = S(3, 0, 0), x2y = S(2, 1, 0), x2z = S(2, 0, 1), xy2 = S(1, 2, 0),
                 xyz = S(1, 1, 1), xz2 = S(1, 0, 2), y3 = S(0, 3, 0), y2z = S(0, 2, 1),
                 yz2 = S(0, 1, 2), z3 = S(0, 0, 3);
    const double x4 = S(4, 0, 0), x3y = S(3, 1, 0), x3z = S(3, 0, 1), x2y2 = S(2, 2, 0),
                 x2yz = S(2, 1, 1), x2z2 = S(2, 0, 2), xy3 = S(1, 3, 0), xy2z = S(1, 2, 1),
                 xyz2 = S(1, 1, 2), xz3 = S(1, 0, 3), y4 = S(0, 4, 0), y3z = S(0, 3, 1),
                 y2z2 = S(0, 2, 2), yz3 = S(0, 1, 3), z4 = S(0, 0, 4);
    const double ri = bmax > 0 ? 1.0 / bmax : 0.0;
    const double tq = (x2 + y2 + z2) / 3.0;
    const double q2[5] = {(x2 - tq) * ri * ri, xy * ri * ri, (y2 - tq) * ri * ri, xz * ri * ri,
                          yz * ri * ri};
    const double tx = (x3 + xy2 + xz2) / 5.0, ty = (x2y + y3 + yz2) / 5.0,
                 tz = (x2z + y2z + z3) / 5.0;
    const double r3 = ri * ri * ri;
    const double q3[7] = {(x3 - 3.0 * tx) * r3, (x2y - ty) * r3, (xy2 - tx) * r3,
                          (y3 - 3.0 * ty) * r3, (x2z - tz) * r3, xyz * r3, (y2z - tz) * r3};
    const double txx = (x4 + x2y2 + x2z2) / 7.0, txy = (x3y + xy3 + xyz2) / 7.0,
                 txz = (x3z + xy2z + xz3) / 7.0, tyy = (x2y2 + y4 + y2z2) / 7.0,
                 tyz = (x2yz + y3z + yz3) / 7.0, tzz = (x2z2 + y2z2 + z4) / 7.0;
    const double tt = 0.1 * (txx + tyy + tzz);
    const double r4 = r3 * ri;
    const double q4[9] = {(x4 - 6.0 * (txx - tt)) * r4, (x3y - 3.0 * txy) * r4,
                          (x2y2 - (txx + tyy - 2.0 * tt)) * r4, (xy3 - 3.0 * txy) * r4,
                          (y4 - 6.0 * (tyy - tt)) * r4, (x3z - 3.0 * txz) * r4,
                          (x2yz - tyz) * r4, (xy2z - txz) * r4, (y3z - 3.0 * tyz) * r4};
    pts[nbodies + c] = make_float4((float)Q[1], (float)Q[2], (float)Q[3], (float)m);
    if (qc) {
        nln_qcell q;
        q.cen[0] = Q[1];
        q.cen[1] = Q[2];
        q.cen[2] = Q[3];
        q.mass = (float)m;
        q.R = (float)bmax;
        q.qxx = (float)q2[0];
        q.qxy = (float)q2[1];
        q.qyy = (float)q2[2];
        q.qxz = (float)q2[3];
        q.qyz = (float)q2[4];
        q.B2 = (float)(x2 + y2 + z2);
        q.pad[0] = q.pad[1] = 0.f;
        qc[c] = q;
    }
    if (hc) {
        nln_hcell h;
        h.cen[0] = Q[1];
        h.cen[1] = Q[2];
        h.cen[2] = Q[3];
        h.mass = (float)m;
        h.R = (float)bmax;
        for (int k = 0; k < 5; k++) h.q2[k] = (float)q2[k];
        for (int k = 0; k < 7; k++) h.q3[k] = (float)q3[k];
        for (int k = 0; k < 9; k++) h.q4[k] = (float)q4[k];
        h.B2 = (float)(x2 + y2 + z2);
        h.pad[0] = h.pad[1] = 0.f;
        hc[c] = h;
    }
}

// Integrate (nln/integrate.c:16-59), COSMO = false: params = {dt, dtv,
// dtsync}; vc = v + dtsync a, v += dtv a, x += dt v.
// CosmoIntegrate (nln/integrate.c:82-135), COSMO = true: params = {kick to
// the positions' time, kick, drift, 1/a0, a1, 1/a0^2}; vc = v + p0 a,
// v += p1 a, x = a1 (x / a0 + drift v) with the reference's three roundings
// to FP32 (its output position is a float written three times), ke scaled
// by 1/a0^2 per body.  Both accumulate energy += {sum m vc.vc, sum m phi};
// positions and velocities are formed in FP64 without fused multiply-adds
// and rounded to FP32, as the reference's double expressions stored to
// floats; m phi is a float product (both operands are floats there).
template <bool COSMO>
__global__ void k_integrate(float4 *__restrict__ pts, const float4 *__restrict__ acc,
                            float4 *__restrict__ vel, int64_t n, const double *__restrict__ params,
                            double *__restrict__ energy) {
    double p[6];
    if (COSMO) {
#pragma unroll
        for (int k = 0; k < 6; k++) p[k] = params[k];
    } else {
        p[0] = params[2];  // dtsync
        p[1] = params[1];  // dtv
        p[2] = params[0];  // dt
        p[3] = p[4] = p[5] = 1.0;
    }
    double ke = 0.0, pe = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        float4 x = pts[i];
        const float4 a = acc[i];
        float4 v = vel[i];
        const double vx = __dadd_rn(v.x, __dmul_rn(p[0], a.x));
        const double vy = __dadd_rn(v.y, __dmul_rn(p[0], a.y));
        const double vz = __dadd_rn(v.z, __dmul_rn(p[0], a.z));
        const double vv = __dadd_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)), __dmul_rn(vz, vz));
        ke = __dadd_rn(ke, COSMO ? __dmul_rn(__dmul_rn((double)x.w, vv), p[5])
                                 : __dmul_rn((double)x.w, vv));
        pe = __dadd_rn(pe, (double)__fmul_rn(x.w, a.w));  // a float product, as the reference's
        v.x = (float)__dadd_rn(v.x, __dmul_rn(p[1], a.x));
        v.y = (float)__dadd_rn(v.y, __dmul_rn(p[1], a.y));
        v.z = (float)__dadd_rn(v.z, __dmul_rn(p[1], a.z));
        if (COSMO) {
            x.x = (float)__dmul_rn(p[3], x.x);
            x.y = (float)__dmul_rn(p[3], x.y);
            x.z = (float)__dmul_rn(p[3], x.z);
        }
        x.x = (float)__dadd_rn(x.x, __dmul_rn(p[2], v.x));
        x.y = (float)__dadd_rn(x.y, __dmul_rn(p[2], v.y));
        x.z = (float)__dadd_rn(x.z, __dmul_rn(p[2], v.z));
        if (COSMO) {
            x.x = (float)__dmul_rn(p[4], x.x);
            x.y = (float)__dmul_rn(p[4], x.y);
            x.z = (float)__dmul_rn(p[4], x.z);
        }
        vel[i] = v;
        pts[i] = x;
    }
    for (int d = 16; d > 0; d >>= 1) {
        ke += __shfl_xor_sync(0xffffffffu, ke, d);
        pe += __shfl_xor_sync(0xffffffffu, pe, d);
    }
    __shared__ double sk[32], sp[32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        sk[w] = ke;
        sp[w] = pe;
    }
    __syncthreads();
    if (w == 0) {
        ke = l < (int)(blockDim.x >> 5) ? sk[l] : 0.0;
        pe = l < (int)(blockDim.x >> 5) ? sp[l] : 0.0;
        for (int d = 16; d > 0; d >>= 1) {
            ke += __shfl_xor_sync(0xffffffffu, ke, d);
            pe += __shfl_xor_sync(0xffffffffu, pe, d);
        }
        if (l == 0) {
            atomicAdd(&energy[0], ke);
            atomicAdd(&energy[1], pe);
        }
    }
}

}  // namespace

// Per-plan state of the time step (owned by the plan, freed with it).
struct grav_step_state {
    cudaMemPool_t pool = nullptr;  // the device buffers came from this pool (adopted links)
    int64_t ncells = 0;
    int64_t *cfirst = nullptr;
    int32_t *ccount = nullptr, *cchild = nullptr, *cnchild = nullptr, *order = nullptr;
    std::vector<int64_t> level_ptr;  // host: cells of depth level, deepest first, in `order`
    double *raw = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    float *graph_vel = nullptr;
    const double *graph_params = nullptr;
    double *graph_energy = nullptr;
    cudaStream_t graph_stream = nullptr;
    ~grav_step_state() {
        if (exec)
            cudaGraphExecDestroy(exec);
        if (graph)
            cudaGraphDestroy(graph);
        for (void *p : {(void *)cfirst, (void *)ccount, (void *)cchild, (void *)cnchild,
                        (void *)order, (void *)raw})
            if (p) {
                if (pool)
                    cudaFreeAsync(p, 0);
                else
                    cudaFree(p);
            }
    }
};

namespace {

int refit_enqueue(grav_plan *pl, cudaStream_t st) {
    grav_step_state *S = pl->step;
    const int64_t nl = (int64_t)S->level_ptr.size() - 1;
    for (int64_t l = 0; l < nl; l++) {
        const int64_t lo = S->level_ptr[l], hi = S->level_ptr[l + 1];
        if (hi <= lo)
            continue;
        k_refit_level<<<(unsigned)((hi - lo + 127) / 128), 128, 0, st>>>(
            pl->dp.points, S->cfirst, S->ccount, S->cchild, S->cnchild, S->order, lo, hi, S->raw);
    }
    k_refit_tables<<<(unsigned)((S->ncells + 127) / 128), 128, 0, st>>>(
        S->raw, S->ncells, pl->hp.nbodies, const_cast<float4 *>(pl->dp.points),
        const_cast<nln_qcell *>(pl->dp.qcells), const_cast<nln_hcell *>(pl->dp.hcells));
    if (pl->qstage || pl->hstage)
        k_stage_cells<<<(unsigned)((S->ncells + 127) / 128), 128, 0, st>>>(
            pl->dp.qcells, pl->dp.hcells, S->ncells, pl->qstage, pl->hstage);
    GC_CHECK(cudaGetLastError());
    return 0;
}

int integrate_enqueue(grav_plan *pl, float *vel, const double *params, double *energy,
                      cudaStream_t st) {
    const int64_t n = pl->hp.nbodies;
    const unsigned blocks = (unsigned)std::min<int64_t>((n + 255) / 256, (int64_t)pl->nsm * 8);
    if (pl->integrator == 1)
        k_integrate<true><<<blocks, 256, 0, st>>>(const_cast<float4 *>(pl->dp.points), pl->dp.out,
                                                  reinterpret_cast<float4 *>(vel), n, params, energy);
    else
        k_integrate<false><<<blocks, 256, 0, st>>>(const_cast<float4 *>(pl->dp.points), pl->dp.out,
                                                   reinterpret_cast<float4 *>(vel), n, params, energy);
    GC_CHECK(cudaGetLastError());
    return 0;
}

int step_enqueue(grav_plan *pl, float *vel, const double *params, double *energy,
                 cudaStream_t st) {
    GC_CHECK(cudaMemsetAsync(energy, 0, 2 * sizeof(double), st));
    if (int rc = grav_groups_eval_CUDA(pl, st))
        return rc;
    if (int rc = integrate_enqueue(pl, vel, params, energy, st))
        return rc;
    return refit_enqueue(pl, st);
}

}  // namespace

void step_state_free(grav_step_state *S) { delete S; }

void step_graph_reset(grav_step_state *S) {
    if (S->exec)
        cudaGraphExecDestroy(S->exec);
    if (S->graph)
        cudaGraphDestroy(S->graph);
    S->exec = nullptr;
    S->graph = nullptr;
}

// The tree links of a plan whose tree was built on the device: the
// builder's device arrays are adopted as they are (no round trip through the
// host), and the per-cell FP64 scratch comes from the same pool.  The
// builder makes cells level by level, so each depth is one index range and
// the deepest-first order is those ranges in reverse; only the depths are
// read back, to find the ranges.  The adopted arrays belong to the plan
// from here on, also when this fails.
int set_tree_adopt(grav_plan *pl, int64_t *cell_first, int32_t *cell_count, int32_t *cell_child,
                   int32_t *cell_nchild, const int32_t *cell_level, cudaMemPool_t pool) {
    const int64_t nc = pl->hp.ncells;
    auto *S = new grav_step_state();
    S->pool = pool;
    S->ncells = nc;
    S->cfirst = cell_first;
    S->ccount = cell_count;
    S->cchild = cell_child;
    S->cnchild = cell_nchild;
    std::vector<int32_t> level((size_t)std::max<int64_t>(nc, 1));
    cudaError_t e = nc > 0 ? cudaMemcpy(level.data(), cell_level, nc * sizeof(int32_t),
                                        cudaMemcpyDeviceToHost)
                           : cudaSuccess;
    if (e != cudaSuccess || nc <= 0) {
        delete S;
        return e != cudaSuccess ? gc::cuda_status(e, "grav_plan_build_CUDA: tree depths")
                                : gc::set_status(-1, "grav_plan_build_CUDA: the plan has no cells");
    }
    std::vector<int64_t> start;  // start[l]: first cell of depth l
    for (int64_t c = 0; c < nc; c++) {
        if (level[c] < 0 || (c > 0 && level[c] < level[c - 1]) || level[c] > (int32_t)start.size()) {
            delete S;
            return gc::set_status(-1, "grav_plan_build_CUDA: cells not in depth order at %lld",
                                  (long long)c);
        }
        if (level[c] == (int32_t)start.size())
            start.push_back(c);
    }
    start.push_back(nc);
    std::vector<int32_t> order;
    order.reserve(nc);
    S->level_ptr.assign(1, 0);
    for (int64_t l = (int64_t)start.size() - 2; l >= 0; l--) {
        for (int64_t c = start[l]; c < start[l + 1]; c++) order.push_back((int32_t)c);
        S->level_ptr.push_back((int64_t)order.size());
    }
    e = cudaMallocFromPoolAsync((void **)&S->order, nc * sizeof(int32_t), pool, 0);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(S->order, order.data(), nc * sizeof(int32_t), cudaMemcpyHostToDevice, 0);
    if (e == cudaSuccess)
        e = cudaMallocFromPoolAsync((void **)&S->raw, (size_t)nc * kRaw * sizeof(double), pool, 0);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(0);  // `order` is read before the host vector goes
    if (e != cudaSuccess) {
        delete S;
        return gc::cuda_status(e, "grav_plan_build_CUDA: tree links");
    }
    delete pl->step;
    pl->step = S;
    return 0;
}

extern "C" int grav_plan_set_tree_CUDA(grav_plan *pl, const int64_t *cell_first,
                                       const int32_t *cell_count, const int32_t *cell_child,
                                       const int32_t *cell_nchild, const int32_t *cell_level) {
    if (!pl || !cell_first || !cell_count || !cell_child || !cell_nchild || !cell_level)
        return gc::set_status(-1, "grav_plan_set_tree_CUDA: bad arguments");
    const int64_t nc = pl->hp.ncells, nb = pl->hp.nbodies;
    if (nc <= 0)
        return gc::set_status(-1, "grav_plan_set_tree_CUDA: the plan has no cells");
    int maxl = 0;
    for (int64_t c = 0; c < nc; c++) {
        const bool leaf = cell_child[c] < 0;
        if (cell_level[c] < 0 || cell_first[c] < 0 || cell_count[c] < 0 ||
            cell_first[c] + cell_count[c] > nb ||
            (!leaf && (cell_child[c] <= c || cell_nchild[c] < 1 || cell_nchild[c] > 8 ||
                       cell_child[c] + cell_nchild[c] > nc)))
            return gc::set_status(-1, "grav_plan_set_tree_CUDA: cell %lld is malformed",
                                  (long long)c);
        if (!leaf)
            for (int32_t k = 0; k < cell_nchild[c]; k++)
                if (cell_level[cell_child[c] + k] != cell_level[c] + 1)
                    return gc::set_status(-1, "grav_plan_set_tree_CUDA: child depth mismatch at "
                                              "cell %lld", (long long)c);
        maxl = std::max(maxl, cell_level[c]);
    }
    // cells by depth, deepest first
    std::vector<int32_t> order;
    order.reserve(nc);
    auto *S = new grav_step_state();
    S->ncells = nc;
    S->level_ptr.assign(1, 0);
    {
        std::vector<std::vector<int32_t>> by(maxl + 1);
        for (int64_t c = 0; c < nc; c++) by[cell_level[c]].push_back((int32_t)c);
        for (int l = maxl; l >= 0; l--) {
            order.insert(order.end(), by[l].begin(), by[l].end());
            S->level_ptr.push_back((int64_t)order.size());
        }
    }
    cudaError_t e = cudaSuccess;
    auto up = [&](auto **dst, const auto *src, size_t n) {
        if (e != cudaSuccess)
            return;
        e = cudaMalloc((void **)dst, n * sizeof(**dst));
        if (e == cudaSuccess)
            e = cudaMemcpy(*dst, src, n * sizeof(**dst), cudaMemcpyHostToDevice);
    };
    up(&S->cfirst, cell_first, nc);
    up(&S->ccount, cell_count, nc);
    up(&S->cchild, cell_child, nc);
    up(&S->cnchild, cell_nchild, nc);
    up(&S->order, order.data(), nc);
    if (e == cudaSuccess)
        e = cudaMalloc((void **)&S->raw, (size_t)nc * kRaw * sizeof(double));
    if (e != cudaSuccess) {
        delete S;
        return gc::cuda_status(e, "grav_plan_set_tree_CUDA");
    }
    delete pl->step;
    pl->step = S;
    return 0;
}

extern "C" int grav_plan_refit_CUDA(grav_plan *pl, void *stream) {
    if (!pl || !pl->step)
        return gc::set_status(-1, "grav_plan_refit_CUDA: no tree links (grav_plan_set_tree_CUDA)");
    return refit_enqueue(pl, (cudaStream_t)stream);
}

extern "C" float *grav_plan_bodies(grav_plan *pl) {
    return pl ? const_cast<float *>(reinterpret_cast<const float *>(pl->dp.points)) : nullptr;
}

extern "C" int grav_plan_set_integrator_CUDA(grav_plan *pl, int kind) {
    if (!pl || kind < 0 || kind > 1)
        return gc::set_status(-1, "grav_plan_set_integrator_CUDA: bad arguments");
    if (pl->integrator != kind && pl->step)
        step_graph_reset(pl->step);
    pl->integrator = kind;
    return 0;
}

extern "C" int grav_plan_integrate_CUDA(grav_plan *pl, float *vel, const double *params,
                                        double *energy, void *stream) {
    if (!pl || !vel || !params || !energy)
        return gc::set_status(-1, "grav_plan_integrate_CUDA: bad arguments");
    return integrate_enqueue(pl, vel, params, energy, (cudaStream_t)stream);
}

extern "C" int grav_plan_step_CUDA(grav_plan *pl, float *vel, const double *params,
                                   double *energy, void *stream, int use_graph) {
    if (!pl || !vel || !params || !energy)
        return gc::set_status(-1, "grav_plan_step_CUDA: bad arguments");
    if (!pl->step)
        return gc::set_status(-1, "grav_plan_step_CUDA: no tree links (grav_plan_set_tree_CUDA)");
    cudaStream_t st = (cudaStream_t)stream;
    if (!use_graph)
        return step_enqueue(pl, vel, params, energy, st);
    if (!st)
        return gc::set_status(-1, "grav_plan_step_CUDA: graph mode needs a created stream");
    grav_step_state *S = pl->step;
    if (S->exec && (S->graph_vel != vel || S->graph_params != params ||
                    S->graph_energy != energy || S->graph_stream != st)) {
        cudaGraphExecDestroy(S->exec);
        cudaGraphDestroy(S->graph);
        S->exec = nullptr;
        S->graph = nullptr;
    }
    if (!S->exec) {
        const int timing = pl->timing;
        pl->timing = 0;  // no event records inside the graph
        GC_CHECK(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
        int rc = step_enqueue(pl, vel, params, energy, st);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(st, &g);
        pl->timing = timing;
        if (rc || e != cudaSuccess) {
            if (g)
                cudaGraphDestroy(g);
            return rc ? rc : gc::cuda_status(e, "grav_plan_step_CUDA: capture");
        }
        e = cudaGraphInstantiate(&S->exec, g, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(g);
            return gc::cuda_status(e, "grav_plan_step_CUDA: instantiate");
        }
        S->graph = g;
        S->graph_vel = vel;
        S->graph_params = params;
        S->graph_energy = energy;
        S->graph_stream = st;
    }
    GC_CHECK(cudaGraphLaunch(S->exec, st));
    return 0;
}
