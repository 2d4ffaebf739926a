// accuracy.cu -- FP64 direct sums at sample sinks: the reference every
// reported force error is measured against.
//
// Isolated: a_i = sum_j m_j d/(r^2+eps2)^1.5, phi_i = -sum_j m_j/(r^2+eps2)^0.5
// with d = x_j - x_i, self included (the scalar do_grav of nln/grav.c:46-79
// summed in FP64).  Periodic: the Ewald-summed direct sum of
// nln/grav_n2.c:97-196 (EwaldForces) with the nearest-image Newtonian term
// Plummer-softened like the tree's: for each pair the nearest-image term
// plus C(y), the smooth remainder of ewald() (nln/ewald.c:13-64), taken from
// an FP64 table over |y_k| <= L/2 by a fifth-order Taylor expansion about
// the nearest node; a pair at zero separation contributes only the constant
// pi/(alpha^2 L^3) that ewald() returns for x = 0.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "gravcuda.h"
#define NLN_EWALD_NO_EXPORT
#include "host/ewald_table.cpp"

namespace {

constexpr double kDirectReach = 0.5;  // min-image displacements
constexpr int kDirectN = 64;

struct Tab64 {
    const double *t;
    int n;
    double h, inv_h;
};

// C and grad C at y from the FP64 table (positive octant, cubic symmetry):
// fifth-order Taylor expansion about the nearest node, C = sum_{|b| <= 5}
// V[b] d^b / b!, dC/dy_i = sum_{|b| <= 4} V[e_i + b] d^b / b!  (multi-index
// layout of nlnlists.h: order n at n(n+1)(n+2)/6, (ax, ay, az) at offset
// (ay+az)(ay+az+1)/2 + az).
__host__ __device__ constexpr int mi(int ax, int ay, int az) {
    return (ax + ay + az) * (ax + ay + az + 1) * (ax + ay + az + 2) / 6 +
           (ay + az) * (ay + az + 1) / 2 + az;
}

__device__ void ew64(const Tab64 &E, double yx, double yy, double yz, double &C, double *G) {
    const double sx = yx < 0 ? -1.0 : 1.0, sy = yy < 0 ? -1.0 : 1.0, sz = yz < 0 ? -1.0 : 1.0;
    const double ax = fabs(yx), ay = fabs(yy), az = fabs(yz);
    const int nm = E.n - 1;
    const int i = min((int)rint(ax * E.inv_h), nm), j = min((int)rint(ay * E.inv_h), nm),
              k = min((int)rint(az * E.inv_h), nm);
    const double d[3] = {ax - i * E.h, ay - j * E.h, az - k * E.h};
    const double *t = E.t + (((size_t)i * E.n + j) * E.n + k) * NLN_EWALD_NQ;
    double p[3][6];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        p[a][0] = 1.0;
#pragma unroll
        for (int q = 1; q < 6; q++) p[a][q] = p[a][q - 1] * d[a] / q;
    }
    double c = 0, g0 = 0, g1 = 0, g2 = 0;
#pragma unroll
    for (int b0 = 0; b0 <= 5; b0++)
#pragma unroll
        for (int b1 = 0; b1 <= 5; b1++)
#pragma unroll
            for (int b2 = 0; b2 <= 5; b2++) {
                if (b0 + b1 + b2 > 5)
                    continue;
                const double w = p[0][b0] * p[1][b1] * p[2][b2];
                c += t[mi(b0, b1, b2)] * w;
                if (b0 + b1 + b2 <= 4) {
                    g0 += t[mi(b0 + 1, b1, b2)] * w;
                    g1 += t[mi(b0, b1 + 1, b2)] * w;
                    g2 += t[mi(b0, b1, b2 + 1)] * w;
                }
            }
    C = c;
    G[0] = sx * g0;
    G[1] = sy * g1;
    G[2] = sz * g2;
}

__global__ void __launch_bounds__(256) k_direct64(const float4 *__restrict__ pts, int64_t n,
                                                  const int64_t *__restrict__ sinks, double eps2,
                                                  double box, Tab64 E, double phi0, double *out) {
    const int64_t i = sinks[blockIdx.x];
    const float4 s = pts[i];
    const double xi = s.x, yi = s.y, zi = s.z;
    double ax = 0, ay = 0, az = 0, ph = 0;
    for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
        const float4 p = pts[j];
        const double m = p.w;
        if (j == i) {
            if (eps2 > 0)
                ph -= m / sqrt(eps2);
            if (box > 0)
                ph += m * phi0;
            continue;
        }
        double dx = (double)p.x - xi, dy = (double)p.y - yi, dz = (double)p.z - zi;
        if (box > 0) {
            dx -= box * rint(dx / box);
            dy -= box * rint(dy / box);
            dz -= box * rint(dz / box);
        }
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (box > 0 && r2 == 0.0) {
            ph += m * phi0;
            if (eps2 > 0)
                ph -= m / sqrt(eps2);
            continue;
        }
        const double rs2 = r2 + eps2;
        if (rs2 == 0.0)
            continue;
        const double ri = 1.0 / sqrt(rs2);
        const double mri = m * ri, mri3 = mri * ri * ri;
        ph -= mri;
        ax += dx * mri3;
        ay += dy * mri3;
        az += dz * mri3;
        if (box > 0) {
            double C, G[3];
            ew64(E, dx, dy, dz, C, G);
            ph += m * C;
            ax += m * G[0];
            ay += m * G[1];
            az += m * G[2];
        }
    }
    __shared__ double red[4][256];
    red[0][threadIdx.x] = ax;
    red[1][threadIdx.x] = ay;
    red[2][threadIdx.x] = az;
    red[3][threadIdx.x] = ph;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int q = 0; q < 4; q++) red[q][threadIdx.x] += red[q][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 4; q++) out[4 * blockIdx.x + q] = red[q][0];
}

}  // namespace

extern "C" int grav_direct_fp64_CUDA(const float *points, int64_t n, const int64_t *sinks,
                                     int64_t nsink, double eps2, double box, double *out) {
    if (!points || n <= 0 || !sinks || nsink <= 0 || !out || eps2 < 0 || box < 0)
        return gc::set_status(-1, "grav_direct_fp64_CUDA: bad arguments");
    for (int64_t k = 0; k < nsink; k++)
        if (sinks[k] < 0 || sinks[k] >= n)
            return gc::set_status(-1, "grav_direct_fp64_CUDA: sink %lld outside the bodies",
                                  (long long)sinks[k]);
    std::vector<void *> alloc;
    auto cleanup = [&]() {
        for (void *p : alloc) cudaFree(p);
    };
    float4 *d_pts = nullptr;
    int64_t *d_s = nullptr;
    double *d_out = nullptr, *d_tab = nullptr;
    cudaError_t e = cudaMalloc(&d_pts, n * sizeof(float4));
    if (e == cudaSuccess) alloc.push_back(d_pts), e = cudaMalloc(&d_s, nsink * sizeof(int64_t));
    if (e == cudaSuccess) alloc.push_back(d_s), e = cudaMalloc(&d_out, nsink * 4 * sizeof(double));
    if (e == cudaSuccess) alloc.push_back(d_out);
    if (e != cudaSuccess) {
        cleanup();
        return gc::cuda_status(e, "grav_direct_fp64_CUDA allocation");
    }
    Tab64 E{nullptr, kDirectN, 0, 0};
    double phi0 = 0;
    if (box > 0) {
        std::vector<double> t((size_t)kDirectN * kDirectN * kDirectN * NLN_EWALD_NQ);
        ewald_table(box, kDirectN, kDirectReach, t.data());
        e = cudaMalloc(&d_tab, t.size() * sizeof(double));
        if (e == cudaSuccess)
            alloc.push_back(d_tab),
                e = cudaMemcpy(d_tab, t.data(), t.size() * sizeof(double), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cleanup();
            return gc::cuda_status(e, "grav_direct_fp64_CUDA table");
        }
        E.t = d_tab;
        E.h = kDirectReach * box / (kDirectN - 1);
        E.inv_h = 1.0 / E.h;
        const double alpha = 2.0 / box;
        phi0 = M_PI / (alpha * alpha * box * box * box);
    }
    e = cudaMemcpy(d_pts, points, n * sizeof(float4), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(d_s, sinks, nsink * sizeof(int64_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_direct64<<<(unsigned)nsink, 256>>>(d_pts, n, d_s, eps2, box, E, phi0, d_out);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(out, d_out, nsink * 4 * sizeof(double), cudaMemcpyDeviceToHost);
    cleanup();
    if (e != cudaSuccess)
        return gc::cuda_status(e, "grav_direct_fp64_CUDA");
    return 0;
}

// ------------------------------------------------------------ FP32 peak
//
// The roofline denominator of the interaction kernels, measured rather than
// derived: every thread runs kChains independent FMA chains x = x * a + b
// (a, b runtime values, so nothing folds), one FMA (2 flops) per chain per
// step, in a grid of blocks_per_sm x SM count blocks of 256 threads.  The
// chains are independent, so the FMA pipes, not the latency, bound it.
// Both forms are timed, scalar fmaf and the paired __ffma2_rn that the
// interaction kernels issue (kChains pairs, twice the FMAs per step), and
// the larger rate is the peak.
namespace {
constexpr int kChains = 8;
constexpr int kPeakThreads = 256;

template <bool PAIRED>
__global__ void __launch_bounds__(kPeakThreads) k_fma_peak(float *out, int iters, float a,
                                                           float b) {
    float s = 0.f;
    if constexpr (PAIRED) {
        float2 x[kChains];
        const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
#pragma unroll
        for (int k = 0; k < kChains; k++)
            x[k] = make_float2((float)(threadIdx.x + k) * 1e-3f, (float)k * 1e-3f);
        for (int i = 0; i < iters; i++) {
#pragma unroll
            for (int u = 0; u < 16; u++)
#pragma unroll
                for (int k = 0; k < kChains; k++) x[k] = __ffma2_rn(x[k], a2, b2);
        }
#pragma unroll
        for (int k = 0; k < kChains; k++) s += x[k].x + x[k].y;
    } else {
        float x[kChains];
#pragma unroll
        for (int k = 0; k < kChains; k++) x[k] = (float)(threadIdx.x + k) * 1e-3f;
        for (int i = 0; i < iters; i++) {
#pragma unroll
            for (int u = 0; u < 16; u++)
#pragma unroll
                for (int k = 0; k < kChains; k++) x[k] = fmaf(x[k], a, b);
        }
#pragma unroll
        for (int k = 0; k < kChains; k++) s += x[k];
    }
    if (s == -1.2345f)  // never true for these inputs; keeps the chains live
        out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}
}  // namespace

extern "C" int grav_fp32_peak_CUDA(double *tflops) {
    if (!tflops)
        return gc::set_status(-1, "grav_fp32_peak_CUDA: bad arguments");
    int dev = 0, nsm = 0;
    GC_CHECK(cudaGetDevice(&dev));
    GC_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = nsm * 8;  // 2048 threads per SM: 64 warps, 16 per scheduler
    const int iters = 4096;      // x 16 x 8 FMAs per thread: ~45 ms per launch on a B200
    float *out = nullptr;
    GC_CHECK(cudaMalloc(&out, (size_t)blocks * kPeakThreads * sizeof(float)));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess)
        e = cudaEventCreate(&e1);
    double best = 0.0;
    for (int paired = 0; paired < 2; paired++)
        for (int rep = 0; rep < 6 && e == cudaSuccess; rep++) {
            e = cudaEventRecord(e0, 0);
            if (e == cudaSuccess) {
                if (paired)
                    k_fma_peak<true><<<blocks, kPeakThreads>>>(out, iters / 2, 0.999f, 1e-4f);
                else
                    k_fma_peak<false><<<blocks, kPeakThreads>>>(out, iters, 0.999f, 1e-4f);
                e = cudaGetLastError();
            }
            if (e == cudaSuccess)
                e = cudaEventRecord(e1, 0);
            if (e == cudaSuccess)
                e = cudaEventSynchronize(e1);
            float ms = 0.f;
            if (e == cudaSuccess)
                e = cudaEventElapsedTime(&ms, e0, e1);
            // a paired step is 2 FMAs per chain; it runs half the steps
            const double flops = 2.0 * kChains * 16.0 * iters * (double)blocks * kPeakThreads;
            if (e == cudaSuccess && rep > 0 && ms > 0.f)  // the first launch warms up
                best = std::max(best, flops / (ms * 1e-3) / 1e12);
        }
    if (e0)
        cudaEventDestroy(e0);
    if (e1)
        cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess)
        return gc::cuda_status(e, "grav_fp32_peak_CUDA");
    *tflops = best;
    return 0;
}
