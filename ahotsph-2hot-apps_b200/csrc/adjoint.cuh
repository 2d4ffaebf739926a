// adjoint.cuh -- the hand-written adjoint of the batched evaluation (no
// counterpart in the reference): for a loss L = sum_i w_i . a_i + u_i phi_i
// on the last evaluation's sinks, dL/dx and dL/dm of every body, with the
// interaction lists held fixed.
//
// Included once, at the end of batch.cu (after step.cuh): it works on the
// plan's tables and uses the tree links of the refit.
//
// Per pair (sink i, source e) with d = x_i - X_e and rho^2 = |d|^2 + eps^2,
// the forward of interact.cuh is phi = -m/rho + qsh rho^-5 d.Q.d (Q the
// staged quadrupole, -3 R^2 q2) and a = -grad_d phi.  With H = grad grad phi
// the pair's loss term -w.grad phi + u phi has
//     dL/dx_i = -(H w + u a) =: -t,     dL/dX_e = +t,
//     dL/dm   = -(w.d rho^-3 + u rho^-1),
//     dL/dQ   = qsh [(u rho^-5 + 5 (w.d) rho^-7) d d^T - rho^-5 (w d^T + d w^T)]
// (the last w.r.t. the full symmetric matrix, Frobenius dual).  Cells pass
// their adjoints to their bodies through M = sum m_b, X = sum m_b x_b / M
// and S2 = sum m_b y_b y_b^T (y_b = x_b - X), with staged Q = -3 (S2 - tr S2/3):
//     dL/dx_b += (m_b/M) Xbar + 2 m_b S2bar y_b,
//     dL/dm_b += Mbar + Xbar.y_b/M + y_b.S2bar.y_b,      S2bar = -3 (Qbar - tr Qbar/3).
//
// Work layout: one warp per work item (group, list kind, slice), as the
// forward's queues.  Lane i holds sink i; a tile's 32 records are staged in
// shared memory and lane i visits record (i + k) mod 32 at step k, so in
// every step the 32 lanes touch 32 different records and accumulate their
// source-side sums into per-record shared slots without conflicts.  Slots
// are flushed with FP64 atomics once per tile; sink sums once per item.
#pragma once

namespace {

constexpr int kAdjTile = 32;
constexpr int kAdjSlot = 11;  // per record: t (3), mass bar, Q bar (6), pad (odd stride)

struct AdjProblem {
    const float4 *points;
    const nln_qcell *qcells;
    const nln_group *groups;
    const uint32_t *list[2];
    const Item *items[2];
    int nitems[2];
    int *counters;
    const float4 *wu;        // (wx, wy, wz, u) per sink, tree order
    double *gbody;           // 4 per body: dL/dx (3), dL/dm
    double *gcell;           // 10 per cell: Mbar, Xbar (3), Qbar (xx xy xz yy yz zz)
    int64_t nbodies;
    float eps2, qsh;
    unsigned *err;
};

template <int KIND>
__global__ void __launch_bounds__(256) k_adjoint(AdjProblem P) {
    constexpr int REC = KIND == KP ? 4 : 12;
    __shared__ __align__(16) float srec[8][kAdjTile * REC];
    __shared__ float sacc[8][kAdjTile * kAdjSlot];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    float *rec = srec[wib];
    float *acc = sacc[wib];
    const uint32_t nb = (uint32_t)P.nbodies;
    while (true) {
        int it = 0;
        if (lane == 0)
            it = atomicAdd(&P.counters[KIND], 1);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= P.nitems[KIND])
            break;
        const Item item = P.items[KIND][it];
        const nln_group G = P.groups[item.group];
        const double c[3] = {G.cen[0], G.cen[1], G.cen[2]};
        float ux = 0.f, uy = 0.f, uz = 0.f, wx = 0.f, wy = 0.f, wz = 0.f, wu = 0.f;
        if (lane < G.count) {
            const float4 s = P.points[G.first + lane];
            ux = (float)((double)s.x - c[0]);
            uy = (float)((double)s.y - c[1]);
            uz = (float)((double)s.z - c[2]);
            const float4 w = P.wu[G.first + lane];
            wx = w.x;
            wy = w.y;
            wz = w.z;
            wu = w.w;
        }
        float gx = 0.f, gy = 0.f, gz = 0.f;  // this sink's -sum t
        for (int64_t b0 = item.begin; b0 < item.end; b0 += kAdjTile) {
            const int nt = (int)min((int64_t)kAdjTile, item.end - b0);
            uint32_t idx = 0;
            if (lane < nt) {
                idx = P.list[KIND][b0 + lane] & NLN_IDX_MASK;
                float *o = rec + lane * REC;
                if (KIND == KP) {
                    const float4 p = P.points[idx];
                    o[0] = (float)((double)p.x - c[0]);
                    o[1] = (float)((double)p.y - c[1]);
                    o[2] = (float)((double)p.z - c[2]);
                    o[3] = p.w;
                } else {
                    const nln_qcell q = P.qcells[idx];
                    o[0] = (float)(q.cen[0] - c[0]);
                    o[1] = (float)(q.cen[1] - c[1]);
                    o[2] = (float)(q.cen[2] - c[2]);
                    o[3] = q.mass;
                    const float q2[5] = {q.qxx, q.qxy, q.qyy, q.qxz, q.qyz};
                    stage_quad(o, q.R, q2);
                }
            }
#pragma unroll
            for (int q = 0; q < kAdjSlot; q++) acc[lane * kAdjSlot + q] = 0.f;
            __syncwarp();
            if (lane < G.count) {
                for (int k = 0; k < kAdjTile; k++) {
                    const int r = (lane + k) & (kAdjTile - 1);
                    if (r >= nt)
                        continue;
                    const float *s = rec + r * REC;
                    const float dx = ux - s[0], dy = uy - s[1], dz = uz - s[2], m = s[3];
                    const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, P.eps2)));
                    const float ri = rsqrt_fast(r2), ri2 = ri * ri, ri3 = ri * ri2;
                    const float wd = fmaf(wx, dx, fmaf(wy, dy, wz * dz));
                    // monopole: t = m (ri3 w - 3 ri5 (w.d) d) - u m ri3 d
                    const float ri5 = ri3 * ri2;
                    const float cd = m * fmaf(-3.f * ri5, wd, -wu * ri3);
                    float tx = fmaf(m * ri3, wx, cd * dx);
                    float ty = fmaf(m * ri3, wy, cd * dy);
                    float tz = fmaf(m * ri3, wz, cd * dz);
                    float* slot = acc + r * kAdjSlot;
                    slot[3] += -fmaf(wd, ri3, wu * ri);  // dL/dm
                    if (KIND == KQ) {
                        const float Qxx = s[4], Qxy = s[5], Qyy = s[6], Qxz = s[7], Qyz = s[8],
                                    Qzz = s[9];
                        const float Qdx = fmaf(Qxx, dx, fmaf(Qxy, dy, Qxz * dz));
                        const float Qdy = fmaf(Qxy, dx, fmaf(Qyy, dy, Qyz * dz));
                        const float Qdz = fmaf(Qxz, dx, fmaf(Qyz, dy, Qzz * dz));
                        const float Qwx = fmaf(Qxx, wx, fmaf(Qxy, wy, Qxz * wz));
                        const float Qwy = fmaf(Qxy, wx, fmaf(Qyy, wy, Qyz * wz));
                        const float Qwz = fmaf(Qxz, wx, fmaf(Qyz, wy, Qzz * wz));
                        const float P2 = fmaf(dx, Qdx, fmaf(dy, Qdy, dz * Qdz));
                        const float Qdw = fmaf(wx, Qdx, fmaf(wy, Qdy, wz * Qdz));
                        const float ri7 = ri5 * ri2, ri9 = ri7 * ri2;
                        const float h = P.qsh;
                        // H_q w = qsh [2 ri5 Qw - 10 ri7 (d (Qd.w) + Qd (d.w)) - 5 ri7 P2 w + 35 ri9 P2 (d.w) d]
                        // a_q = -qsh [2 ri5 Qd - 5 ri7 P2 d]
                        const float kd = h * (-10.f * ri7 * Qdw + 35.f * ri9 * P2 * wd + 5.f * wu * ri7 * P2);
                        const float kq = h * (-10.f * ri7 * wd - 2.f * wu * ri5);
                        const float kw = h * (-5.f * ri7 * P2);
                        const float k2 = h * 2.f * ri5;
                        tx += fmaf(k2, Qwx, fmaf(kd, dx, fmaf(kq, Qdx, kw * wx)));
                        ty += fmaf(k2, Qwy, fmaf(kd, dy, fmaf(kq, Qdy, kw * wy)));
                        tz += fmaf(k2, Qwz, fmaf(kd, dz, fmaf(kq, Qdz, kw * wz)));
                        // dL/dQ = qsh [(u ri5 + 5 (w.d) ri7) d d^T - ri5 (w d^T + d w^T)]
                        const float A = h * fmaf(wu, ri5, 5.f * wd * ri7);
                        const float B = -h * ri5;
                        slot[4] += fmaf(A * dx, dx, 2.f * B * wx * dx);
                        slot[5] += fmaf(A * dx, dy, B * fmaf(wx, dy, wy * dx));
                        slot[6] += fmaf(A * dx, dz, B * fmaf(wx, dz, wz * dx));
                        slot[7] += fmaf(A * dy, dy, 2.f * B * wy * dy);
                        slot[8] += fmaf(A * dy, dz, B * fmaf(wy, dz, wz * dy));
                        slot[9] += fmaf(A * dz, dz, 2.f * B * wz * dz);
                    }
                    slot[0] += tx;
                    slot[1] += ty;
                    slot[2] += tz;
                    gx -= tx;
                    gy -= ty;
                    gz -= tz;
                }
            }
            __syncwarp();
            if (lane < nt) {
                const float *slot = acc + lane * kAdjSlot;
                if (KIND == KP && idx < nb) {
                    double *g = P.gbody + (size_t)idx * 4;
                    atomicAdd(g + 0, (double)slot[0]);
                    atomicAdd(g + 1, (double)slot[1]);
                    atomicAdd(g + 2, (double)slot[2]);
                    atomicAdd(g + 3, (double)slot[3]);
                } else {
                    const uint32_t ci = KIND == KP ? idx - nb : idx;
                    double *g = P.gcell + (size_t)ci * 10;
                    atomicAdd(g + 0, (double)slot[3]);
                    atomicAdd(g + 1, (double)slot[0]);
                    atomicAdd(g + 2, (double)slot[1]);
                    atomicAdd(g + 3, (double)slot[2]);
                    if (KIND == KQ)
                        for (int q = 0; q < 6; q++) atomicAdd(g + 4 + q, (double)slot[4 + q]);
                }
            }
            __syncwarp();  // the staged records are reused by the next tile
        }
        if (lane < G.count) {
            double *g = P.gbody + (size_t)(G.first + lane) * 4;
            atomicAdd(g + 0, (double)gx);
            atomicAdd(g + 1, (double)gy);
            atomicAdd(g + 2, (double)gz);
        }
    }
}

// Bodies from their cells' adjoints: every ancestor of the body's leaf.
// A cell's centre and mass are read as the forward used them: the FP64
// centre of the quadrupole table when there is one, else the cell monopole
// of the point table.
__global__ void k_adjoint_bodies(const float4 *__restrict__ pts, const int32_t *__restrict__ leaf,
                                 const int32_t *__restrict__ parent, const nln_qcell *__restrict__ qc,
                                 const double *__restrict__ gcell, const double *__restrict__ gbody,
                                 int64_t n, float4 *__restrict__ out) {
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n)
        return;
    const float4 p = pts[b];
    double g[4] = {gbody[4 * b], gbody[4 * b + 1], gbody[4 * b + 2], gbody[4 * b + 3]};
    for (int32_t cidx = leaf[b]; cidx >= 0; cidx = parent[cidx]) {
        const double *A = gcell + (size_t)cidx * 10;
        if (A[0] == 0.0 && A[1] == 0.0 && A[2] == 0.0 && A[3] == 0.0 && A[4] == 0.0 &&
            A[5] == 0.0 && A[6] == 0.0 && A[7] == 0.0 && A[8] == 0.0 && A[9] == 0.0)
            continue;
        double X[3], M;
        if (qc) {
            X[0] = qc[cidx].cen[0];
            X[1] = qc[cidx].cen[1];
            X[2] = qc[cidx].cen[2];
            M = qc[cidx].mass;
        } else {
            const float4 cm = pts[n + cidx];
            X[0] = cm.x;
            X[1] = cm.y;
            X[2] = cm.z;
            M = cm.w;
        }
        if (M == 0.0)
            continue;
        const double y[3] = {(double)p.x - X[0], (double)p.y - X[1], (double)p.z - X[2]};
        // S2bar = -3 (Qbar - tr Qbar / 3)
        const double tr = (A[4] + A[7] + A[9]) / 3.0;
        const double S[6] = {-3.0 * (A[4] - tr), -3.0 * A[5], -3.0 * A[6], -3.0 * (A[7] - tr),
                             -3.0 * A[8], -3.0 * (A[9] - tr)};
        const double Sy[3] = {S[0] * y[0] + S[1] * y[1] + S[2] * y[2],
                              S[1] * y[0] + S[3] * y[1] + S[4] * y[2],
                              S[2] * y[0] + S[4] * y[1] + S[5] * y[2]};
        const double mb = p.w;
        for (int d = 0; d < 3; d++) g[d] += (mb / M) * A[1 + d] + 2.0 * mb * Sy[d];
        g[3] += A[0] + (A[1] * y[0] + A[2] * y[1] + A[3] * y[2]) / M +
                (y[0] * Sy[0] + y[1] * Sy[1] + y[2] * Sy[2]);
    }
    out[b] = make_float4((float)g[0], (float)g[1], (float)g[2], (float)g[3]);
}

}  // namespace

// Per-plan adjoint state (owned by the plan).
struct grav_adjoint_state {
    int32_t *leaf = nullptr, *parent = nullptr;
    double *gbody = nullptr, *gcell = nullptr;
    ~grav_adjoint_state() {
        for (void *p : {(void *)leaf, (void *)parent, (void *)gbody, (void *)gcell})
            if (p)
                cudaFree(p);
    }
};

void adjoint_state_free(grav_adjoint_state *A) { delete A; }

extern "C" int grav_plan_adjoint_CUDA(grav_plan *pl, const float *wu, float *grad, void *stream) {
    if (!pl || !wu || !grad)
        return gc::set_status(-1, "grav_plan_adjoint_CUDA: bad arguments");
    if (!pl->step)
        return gc::set_status(-1, "grav_plan_adjoint_CUDA: no tree links (grav_plan_set_tree_CUDA)");
    if (pl->hp.box > 0 || pl->dp.nitems[KH] > 0)
        return gc::set_status(-1, "grav_plan_adjoint_CUDA: isolated problems with monopole and "
                                  "quadrupole lists only (no order-4 cells, no periodic images)");
    if (pl->dp.nitems[KQ] > 0 && !pl->dp.qcells)
        return gc::set_status(-1, "grav_plan_adjoint_CUDA: no quadrupole table");
    if (pl->dp.qsh != 0.5f)
        return gc::set_status(-1, "grav_plan_adjoint_CUDA: the physical quadrupole potential "
                                  "(quad_phi_sign = +1) only");
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t nb = pl->hp.nbodies, nc = pl->hp.ncells;
    grav_step_state *S = pl->step;
    if (!pl->adj) {
        auto *A = new grav_adjoint_state();
        // leaf of every body and parent of every cell, from the links
        std::vector<int32_t> child(nc), nchild(nc), parent(nc, -1), leaf(nb, -1);
        std::vector<int64_t> first(nc);
        std::vector<int32_t> count(nc);
        cudaError_t e = cudaMemcpy(child.data(), S->cchild, nc * 4, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess)
            e = cudaMemcpy(nchild.data(), S->cnchild, nc * 4, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess)
            e = cudaMemcpy(first.data(), S->cfirst, nc * 8, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess)
            e = cudaMemcpy(count.data(), S->ccount, nc * 4, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            delete A;
            return gc::cuda_status(e, "grav_plan_adjoint_CUDA: links");
        }
        for (int64_t c = 0; c < nc; c++) {
            if (child[c] >= 0) {
                for (int32_t k = 0; k < nchild[c]; k++) parent[child[c] + k] = (int32_t)c;
            } else {
                for (int64_t b = first[c]; b < first[c] + count[c]; b++) leaf[b] = (int32_t)c;
            }
        }
        e = cudaMalloc((void **)&A->leaf, nb * 4);
        if (e == cudaSuccess)
            e = cudaMemcpy(A->leaf, leaf.data(), nb * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMalloc((void **)&A->parent, nc * 4);
        if (e == cudaSuccess)
            e = cudaMemcpy(A->parent, parent.data(), nc * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMalloc((void **)&A->gbody, nb * 4 * sizeof(double));
        if (e == cudaSuccess)
            e = cudaMalloc((void **)&A->gcell, nc * 10 * sizeof(double));
        if (e != cudaSuccess) {
            delete A;
            return gc::cuda_status(e, "grav_plan_adjoint_CUDA: scratch");
        }
        pl->adj = A;
    }
    grav_adjoint_state *A = pl->adj;
    GC_CHECK(cudaMemsetAsync(A->gbody, 0, nb * 4 * sizeof(double), st));
    GC_CHECK(cudaMemsetAsync(A->gcell, 0, nc * 10 * sizeof(double), st));
    GC_CHECK(cudaMemsetAsync(pl->dp.counters, 0, 4 * sizeof(int), st));
    AdjProblem P{};
    P.points = pl->dp.points;
    P.qcells = pl->dp.qcells;
    P.groups = pl->dp.groups;
    P.list[0] = pl->dp.list[KP];
    P.list[1] = pl->dp.list[KQ];
    P.items[0] = pl->dp.items[KP];
    P.items[1] = pl->dp.items[KQ];
    P.nitems[0] = pl->dp.nitems[KP];
    P.nitems[1] = pl->dp.nitems[KQ];
    P.counters = pl->dp.counters;
    P.wu = reinterpret_cast<const float4 *>(wu);
    P.gbody = A->gbody;
    P.gcell = A->gcell;
    P.nbodies = nb;
    P.eps2 = pl->dp.eps2;
    P.qsh = pl->dp.qsh;
    P.err = pl->dp.err;
    const unsigned blocks = (unsigned)pl->nsm * 4;
    if (P.nitems[0] > 0)
        k_adjoint<KP><<<blocks, 256, 0, st>>>(P);
    if (P.nitems[1] > 0)
        k_adjoint<KQ><<<blocks, 256, 0, st>>>(P);
    GC_CHECK(cudaGetLastError());
    k_adjoint_bodies<<<(unsigned)((nb + 255) / 256), 256, 0, st>>>(
        pl->dp.points, A->leaf, A->parent, pl->dp.qcells, A->gcell, A->gbody, nb,
        reinterpret_cast<float4 *>(grad));
    GC_CHECK(cudaGetLastError());
    return 0;
}
