// dropin.cu -- Part 1 of gravcuda.h: the reference entry points
// (nln/gravcuda.h:13-69) on B200.
//
// Differences in mechanism from nln/pgrav.cu (semantics are kept):
//  * 32 queue slots with persistent streams and growable pinned/device
//    buffers (the reference created a stream per call and aborted above 1 MB);
//  * list tiles are staged into shared memory by double-buffered TMA bulk
//    copies (cp.async.bulk + mbarrier), folded once per source, and read by
//    every thread of the block as broadcasts;
//  * a long list is split across blocks (grid.y) and each thread holds
//    SPT sinks, so one call fills more than a handful of SMs;
//  * results are accumulated with one float4 atomic per sink per block;
//  * grav_mn_CUDA returns once the list is copied out of the caller's
//    memory into page-locked staging; a submitter thread issues the copy to
//    the device and the launch, so the caller's next list copy overlaps the
//    CUDA calls of this one.
#include <cuda_runtime.h>
#include <immintrin.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "gravcuda.h"
#include "interact.cuh"

// ------------------------------------------------------------ status
namespace gc {
int g_error_mode = 0;
static int g_status = 0;
static std::string g_status_msg;
static std::mutex g_status_mu;

int set_status(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    {
        std::lock_guard<std::mutex> lk(g_status_mu);
        g_status = code;
        g_status_msg = buf;
    }
    if (g_error_mode == 0) {
        fprintf(stderr, "gravcuda error %d: %s\n", code, buf);
        abort();
    }
    return code;
}

int cuda_status(cudaError_t err, const char *what) {
    return set_status((int)err, "%s: %s", what, cudaGetErrorString(err));
}
}  // namespace gc

extern "C" void gravcuda_set_error_mode(int mode) { gc::g_error_mode = mode ? 1 : 0; }
extern "C" int gravcuda_status(void) { return gc::g_status; }
extern "C" const char *gravcuda_status_string(void) { return gc::g_status_msg.c_str(); }
extern "C" void gravcuda_clear_status(void) {
    std::lock_guard<std::mutex> lk(gc::g_status_mu);
    gc::g_status = 0;
    gc::g_status_msg.clear();
}

// ------------------------------------------------------------ kernels
namespace {

constexpr int NQ = 32;          // queue slots (nln/pgrav.cu:812)
constexpr int SPT = 2;          // sinks per thread
constexpr int TBLK = 8;         // 8-lane list blocks per staged tile (64 sources)
constexpr int TSRC = TBLK * 8;

template <int ORDER>
struct RecOf {
    static constexpr int v = ORDER == 0 ? REC_P : (ORDER == 2 ? REC_Q : REC_H);
};

// Fold source s of a raw AoSoA tile (sz fields x 8 lanes per block) into a
// staged record.  Zero-mass padding lanes (nln/mac.c:606-612) are moved far
// away so they add exactly zero even without softening; 1e8 keeps every
// power of the displacement used by the order-4 terms (up to the 4th) finite.
constexpr float kFarAway = 1.0e8f;

template <int ORDER>
__device__ void stage_aosoa(float *o, const float *raw, int sz, int s) {
    const float *blk = raw + (s >> 3) * sz * 8;
    const int l = s & 7;
    float m = blk[l];
    float x = blk[8 + l], y = blk[16 + l], z = blk[24 + l];
    if (m == 0.0f) {
        x = y = z = kFarAway;
    }
    o[0] = x;
    o[1] = y;
    o[2] = z;
    o[3] = m;
    if (ORDER >= 2) {
        float R = blk[4 * 8 + l];
        float q2[5];
#pragma unroll
        for (int k = 0; k < 5; k++) q2[k] = blk[(8 + k) * 8 + l];
        stage_quad(o, R, q2);
        if (ORDER >= 4) {
            float q3[7], q4[9];
#pragma unroll
            for (int k = 0; k < 7; k++) q3[k] = blk[(13 + k) * 8 + l];
#pragma unroll
            for (int k = 0; k < 9; k++) q4[k] = blk[(20 + k) * 8 + l];
            stage_hexa(o, R, q3, q4);
        }
    }
}

// Sinks [base_sink, base_sink+m) against list blocks [c0, c1) of f, c0/c1
// from blockIdx.y.  Dynamic shared memory: 2 raw tiles + staged records + 2 mbarriers.
template <int ORDER, int SOFT>
__global__ void __launch_bounds__(128) k_list(const float *__restrict__ pos, float4 *accp, int m,
                                              const float *__restrict__ f, int nblk, int sz,
                                              int blk_per_chunk, float e, float qsh,
                                              unsigned *err) {
    constexpr int REC = RecOf<ORDER>::v;
    extern __shared__ __align__(128) unsigned char smem[];
    const int raw_floats = TBLK * sz * 8;
    float *raw0 = reinterpret_cast<float *>(smem);
    float *raw1 = raw0 + raw_floats;
    float *rec = raw1 + raw_floats;
    uint64_t *bar = reinterpret_cast<uint64_t *>(rec + TSRC * REC);

    const int c0 = blockIdx.y * blk_per_chunk;
    const int c1 = min(nblk, c0 + blk_per_chunk);
    const int ntile = (c1 - c0 + TBLK - 1) / TBLK;
    const int tid = threadIdx.x;

    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int t) {
        int b0 = c0 + t * TBLK;
        int nb = min(TBLK, c1 - b0);
        uint32_t bytes = (uint32_t)nb * sz * 8 * 4;
        float *dst = (t & 1) ? raw1 : raw0;
        mbar_arrive_expect_tx(&bar[t & 1], bytes);
        tma_bulk_g2s(dst, f + (size_t)b0 * sz * 8, bytes, &bar[t & 1]);
    };
    if (tid == 0 && ntile > 0)
        issue(0);

    float sx[SPT], sy[SPT], sz_[SPT];
    Acc4 a[SPT];
    int idx[SPT];
#pragma unroll
    for (int k = 0; k < SPT; k++) {
        idx[k] = blockIdx.x * blockDim.x * SPT + k * blockDim.x + tid;
        int i = min(idx[k], m - 1);
        sx[k] = pos[3 * i];
        sy[k] = pos[3 * i + 1];
        sz_[k] = pos[3 * i + 2];
        a[k] = Acc4{0.f, 0.f, 0.f, 0.f};
    }

    bool ok = true;
    int failed_at = -1;
    for (int t = 0; t < ntile; t++) {
        if (tid == 0 && t + 1 < ntile)
            issue(t + 1);
        ok = mbar_wait_bounded(&bar[t & 1], (t >> 1) & 1, err);
        if (!__syncthreads_and(ok)) {
            ok = false;
            failed_at = t;
            break;
        }
        const float *rt = (t & 1) ? raw1 : raw0;
        const int nsrc = min(TBLK, c1 - (c0 + t * TBLK)) * 8;
        for (int s = tid; s < nsrc; s += blockDim.x) stage_aosoa<ORDER>(rec + s * REC, rt, sz, s);
        __syncthreads();
        for (int s = 0; s < nsrc; s++) {
            const float *r = rec + s * REC;
#pragma unroll
            for (int k = 0; k < SPT; k++) interact<ORDER, SOFT>(r, sx[k], sy[k], sz_[k], e, qsh, a[k]);
        }
        __syncthreads();
    }
    if (!ok) {
        // drain: wait (bounded) for the next tile's copy, if one was issued
        const int t1 = failed_at + 1;
        if (tid == 0 && t1 < ntile)
            mbar_wait_bounded(&bar[t1 & 1], (t1 >> 1) & 1, err, 1u << 16);
        return;
    }
#pragma unroll
    for (int k = 0; k < SPT; k++)
        if (idx[k] < m)
            atomicAdd(&accp[idx[k]], make_float4(a[k].ax, a[k].ay, a[k].az, a[k].phi));
}

// Body-run p-p with K1 softening, one thread per sink, runs read through
// the read-only cache (pMM1_mnss_sK1, nln/pgrav.cu:713-790).  group_of
// maps sink -> group (NULL: one group for all), runs of group g are
// seg[gs[g].base .. +gs[g].length).
__global__ void k_runs_k1(const float *__restrict__ pos, float4 *accp, int m,
                          const uint16_t *__restrict__ group_of, const segment *__restrict__ gs,
                          const segment *__restrict__ seg, int seg_total,
                          const float *__restrict__ src, int nsrc_total,
                          const int *__restrict__ expect, float mass, float e, unsigned *err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m)
        return;
    const int g = group_of ? group_of[i] : 0;
    const segment r = gs[g];
    float sx = pos[3 * i], sy = pos[3 * i + 1], sz = pos[3 * i + 2];
    Acc4 a{0.f, 0.f, 0.f, 0.f};
    long count = 0;
    for (unsigned k = 0; k < r.length; k++) {
        if ((int)(r.base + k) >= seg_total) {
            atomicOr(err, GC_DEV_BAD_INDEX);
            break;
        }
        const segment s = seg[r.base + k];
        if ((long)s.base + s.length > nsrc_total) {
            atomicOr(err, GC_DEV_BAD_INDEX);
            break;
        }
        count += s.length;
        for (unsigned j = 0; j < s.length; j++) {
            const float *q = src + 3 * (size_t)(s.base + j);
            float x = sx - __ldg(q), y = sy - __ldg(q + 1), z = sz - __ldg(q + 2);
            float ri, ri2;
            mono<SOFT_K1>(x, y, z, mass, e, a, ri, ri2);
        }
    }
    if (expect && count != expect[g])
        atomicOr(err, GC_DEV_BAD_COUNT);
    atomicAdd(&accp[i], make_float4(a.ax, a.ay, a.az, a.phi));
}

// Quadrupole (no softening, reference sign -1) of every sink in [0, m)
// against per-sink runs of a packed QSZ AoSoA buffer (pQ1_mnss,
// nln/pgrav.cu:293-368) or against the cell table by index (pQQ1,
// nln/pgrav.cu:498-572).  One thread per sink; records staged per thread.
// The dipole term of do_gravdq_avx8 (nln/do_grav_avx8.c:428-436) and of the
// CUDA pQ1_mnss / pQQ1 kernels (nln/pgrav.cu:334-344,534-544), for a record
// whose expansion centre is not its centre of mass: with d = sink - source,
// t = -R / r^3, eq = t q:  phi += eq.d,  a += 3 d (eq.d) / r^2 - eq.
__device__ __forceinline__ void dipole_term(float dx, float dy, float dz, float R, float qx,
                                            float qy, float qz, Acc4 &a) {
    const float r2 = dx * dx + dy * dy + dz * dz;
    const float rinv = rsqrtf(r2);
    const float rinv2 = rinv * rinv;
    const float t = -R * rinv * rinv2;
    const float e0 = t * qx, e1 = t * qy, e2 = t * qz;
    float ed = dx * e0 + dy * e1 + dz * e2;
    a.phi += ed;
    ed *= 3.0f * rinv2;
    a.ax += dx * ed - e0;
    a.ay += dy * ed - e1;
    a.az += dz * ed - e2;
}

__global__ void k_quad_runs(const float *__restrict__ pos, float4 *accp, int m,
                            const segment *__restrict__ seg, const float *__restrict__ src,
                            int nsrc, unsigned *err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m)
        return;
    const segment s = seg[i];
    if ((long)s.base + s.length > nsrc) {
        atomicOr(err, GC_DEV_BAD_INDEX);
        return;
    }
    float sx = pos[3 * i], sy = pos[3 * i + 1], sz = pos[3 * i + 2];
    Acc4 a{0.f, 0.f, 0.f, 0.f};
    float rec[REC_Q];
    for (unsigned k = 0; k < s.length; k++) {
        const unsigned j = s.base + k;
        const float *blk = src + (size_t)(j >> 3) * 13 * 8;
        const int l = j & 7;
        float mm = __ldg(blk + l);
        rec[0] = __ldg(blk + 8 + l);
        rec[1] = __ldg(blk + 16 + l);
        rec[2] = __ldg(blk + 24 + l);
        rec[3] = mm;
        if (mm == 0.0f)
            rec[0] = rec[1] = rec[2] = kFarAway;
        float q2[5];
        for (int t = 0; t < 5; t++) q2[t] = __ldg(blk + (8 + t) * 8 + l);
        const float R = __ldg(blk + 32 + l);
        stage_quad(rec, R, q2);
        interact<2, SOFT_NONE>(rec, sx, sy, sz, 0.0f, -0.5f, a);
        if (mm != 0.0f)
            dipole_term(sx - rec[0], sy - rec[1], sz - rec[2], R, __ldg(blk + 40 + l),
                        __ldg(blk + 48 + l), __ldg(blk + 56 + l), a);
    }
    atomicAdd(&accp[i], make_float4(a.ax, a.ay, a.az, a.phi));
}

__global__ void k_quad_index(const float *__restrict__ pos, float4 *accp, int m,
                             const int *__restrict__ list, int nlist,
                             const float *__restrict__ qtab, int ncells, unsigned *err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m)
        return;
    float sx = pos[3 * i], sy = pos[3 * i + 1], sz = pos[3 * i + 2];
    Acc4 a{0.f, 0.f, 0.f, 0.f};
    float rec[REC_Q];
    for (int k = 0; k < nlist; k++) {
        int c = list[k];
        if (c < 0 || c >= ncells) {
            atomicOr(err, GC_DEV_BAD_INDEX);
            continue;
        }
        const float *q = qtab + (size_t)c * 13;  // m x y z R qxx qxy qyy qxz qyz qx qy qz
        rec[0] = __ldg(q + 1);
        rec[1] = __ldg(q + 2);
        rec[2] = __ldg(q + 3);
        rec[3] = __ldg(q);
        float q2[5];
        for (int t = 0; t < 5; t++) q2[t] = __ldg(q + 5 + t);
        const float R = __ldg(q + 4);
        stage_quad(rec, R, q2);
        interact<2, SOFT_NONE>(rec, sx, sy, sz, 0.0f, -0.5f, a);
        dipole_term(sx - rec[0], sy - rec[1], sz - rec[2], R, __ldg(q + 10), __ldg(q + 11),
                    __ldg(q + 12), a);
    }
    atomicAdd(&accp[i], make_float4(a.ax, a.ay, a.az, a.phi));
}

// ------------------------------------------------------------ state
// A queue slot: its stream, a device list buffer, and two page-locked
// staging buffers used in turn; the copy out of each staging buffer records
// an event, so reusing a staging buffer waits only for the copy that last
// read it (two calls back), never for the slot's kernels.
struct Slot {
    bool inuse = false;
    cudaStream_t stream = nullptr;
    size_t cap = 0;
    void *host = nullptr;      // the staging buffer of the current call
    void *hbuf[2] = {nullptr, nullptr};
    cudaEvent_t copied[2] = {nullptr, nullptr};
    // staging buffer states: 0 free, 1 filled and waiting for the submitter,
    // 2 its copy to the device issued (copied[k] recorded)
    std::atomic<int> bstate[2] = {{0}, {0}};
    std::atomic<int> queued{0};  // jobs of this slot not yet issued
    // recorded by the submitter after each launch; kpending = 1 until the
    // submitter has seen it complete (then qallocCUDA needs no stream query)
    cudaEvent_t kdone = nullptr;
    std::atomic<int> kpending{0};
    int turn = 0;
    void *dev = nullptr;
    void reset() {
        kdone = nullptr;
        kpending.store(0);
        inuse = false;
        stream = nullptr;
        cap = 0;
        host = nullptr;
        for (int k = 0; k < 2; k++) {
            hbuf[k] = nullptr;
            copied[k] = nullptr;
            bstate[k].store(0);
        }
        queued.store(0);
        turn = 0;
        dev = nullptr;
    }
};

struct State {
    bool init = false;
    Slot q[NQ];
    float *Btab = nullptr;
    int bstride = 0;
    int64_t nobj = 0;
    float *devpos = nullptr;     // 3 floats per sink
    float4 *devaccp = nullptr;   // ax ay az phi per sink
    float *qdev = nullptr;       // cell table for pQQ1, 10 floats per cell
    int64_t ncells = 0;
    unsigned *derr = nullptr;    // device error word
    int nsm = 148;
};
State S;
// The entry points that use the slots run one at a time (nln/mac.c calls
// them from one thread; this makes concurrent callers safe too).
std::recursive_mutex g_call_mu;

// Seconds spent per phase of the drop-in calls since the last
// WalkInitSinkCUDA (gravcuda_dropin_phases): copies into staging, waits for
// a free staging buffer, waits for room in the submitter's queue, the
// submitter's CUDA calls, the drain at WalkTerminateSinkCUDA; and the calls.
std::atomic<int64_t> g_phase_ns[5] = {{0}, {0}, {0}, {0}, {0}};
std::atomic<int64_t> g_phase_calls{0};
inline int64_t now_ns() {
    return std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

int ensure_init() {
    if (S.init)
        return 0;
    GC_CHECK(cudaSetDevice(0));
    GC_CHECK(cudaMalloc(&S.derr, sizeof(unsigned)));
    GC_CHECK(cudaMemset(S.derr, 0, sizeof(unsigned)));
    cudaDeviceGetAttribute(&S.nsm, cudaDevAttrMultiProcessorCount, 0);
    for (int i = 0; i < NQ; i++) {
        GC_CHECK(cudaStreamCreateWithFlags(&S.q[i].stream, cudaStreamNonBlocking));
        GC_CHECK(cudaEventCreateWithFlags(&S.q[i].kdone, cudaEventDisableTiming));
    }
    S.init = true;
    return 0;
}

// Wait, with a bound, until `done` holds; false when the bound ran out.
template <typename F>
bool wait_until(F done, double seconds = 120.0) {
    const auto t0 = std::chrono::steady_clock::now();
    for (int spin = 0; !done(); spin++) {
        if (spin < 4096)
            continue;
        std::this_thread::yield();
        if ((spin & 1023) == 0 &&
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > seconds)
            return false;
    }
    return true;
}

// Make slot q ready for a call of `bytes`: staging buffer s.host free to
// write (the copy that last read it has been issued and has completed),
// device buffer large enough.  The device buffer is only rewritten by copies
// on the slot's own stream, which run after the kernels queued before them.
int slot_reserve(int q, size_t bytes) {
    if (q < 0 || q >= NQ)
        return gc::set_status(-1, "queue slot %d out of range", q);
    Slot &s = S.q[q];
    if (s.cap < bytes) {
        if (!wait_until([&] { return s.queued.load(std::memory_order_acquire) == 0; }))
            return gc::set_status(-1, "queue slot %d: the submitter did not drain", q);
        GC_CHECK(cudaStreamSynchronize(s.stream));
        for (int k = 0; k < 2; k++) {
            if (s.hbuf[k])
                GC_CHECK(cudaFreeHost(s.hbuf[k]));
            s.hbuf[k] = nullptr;
            s.bstate[k].store(0);
            if (!s.copied[k])
                GC_CHECK(cudaEventCreateWithFlags(&s.copied[k], cudaEventDisableTiming));
        }
        if (s.dev)
            GC_CHECK(cudaFree(s.dev));
        size_t cap = 1 << 20;
        while (cap < bytes) cap <<= 1;
        for (int k = 0; k < 2; k++) GC_CHECK(cudaMallocHost(&s.hbuf[k], cap));
        GC_CHECK(cudaMalloc(&s.dev, cap));
        s.cap = cap;
    }
    s.turn ^= 1;
    std::atomic<int> &st = s.bstate[s.turn];
    const int64_t t0 = now_ns();
    if (!wait_until([&] { return st.load(std::memory_order_acquire) != 1; }))
        return gc::set_status(-1, "queue slot %d: the submitter did not issue", q);
    if (st.load(std::memory_order_acquire) == 2) {
        GC_CHECK(cudaEventSynchronize(s.copied[s.turn]));
        st.store(0, std::memory_order_relaxed);
    }
    g_phase_ns[1] += now_ns() - t0;
    s.host = s.hbuf[s.turn];
    return 0;
}

// The synchronous form (the body-run and index-list entry points): issue
// the copy from the calling thread after every queued job of the slot.
int slot_copied(Slot &s) {
    GC_CHECK(cudaEventRecord(s.copied[s.turn], s.stream));
    s.bstate[s.turn].store(2, std::memory_order_release);
    return 0;
}

int slot_quiet(int q) {
    if (!wait_until([&] { return S.q[q].queued.load(std::memory_order_acquire) == 0; }))
        return gc::set_status(-1, "queue slot %d: the submitter did not drain", q);
    return 0;
}

// Streaming copy into page-locked memory: non-temporal 32-byte stores
// write the destination without reading it into the caches first, which a
// plain memcpy of a few hundred KB does (glibc streams only far larger
// copies).  The fence makes the stores visible before the copy is reported
// done, to other threads and to the device copy that reads the buffer.
__attribute__((target("avx2"))) void stream_copy_avx2(char *d, const char *s, size_t n) {
    size_t i = 0;
    for (; i + 128 <= n; i += 128) {
        const __m256i x0 = _mm256_loadu_si256(reinterpret_cast<const __m256i *>(s + i));
        const __m256i x1 = _mm256_loadu_si256(reinterpret_cast<const __m256i *>(s + i + 32));
        const __m256i x2 = _mm256_loadu_si256(reinterpret_cast<const __m256i *>(s + i + 64));
        const __m256i x3 = _mm256_loadu_si256(reinterpret_cast<const __m256i *>(s + i + 96));
        _mm256_stream_si256(reinterpret_cast<__m256i *>(d + i), x0);
        _mm256_stream_si256(reinterpret_cast<__m256i *>(d + i + 32), x1);
        _mm256_stream_si256(reinterpret_cast<__m256i *>(d + i + 64), x2);
        _mm256_stream_si256(reinterpret_cast<__m256i *>(d + i + 96), x3);
    }
    if (i < n)
        memcpy(d + i, s + i, n - i);
    _mm_sfence();
}

void copy_bytes(char *d, const char *s, size_t n) {
    static const bool avx2 = __builtin_cpu_supports("avx2");
    if (avx2 && n >= 4096 && ((uintptr_t)d & 31) == 0)
        stream_copy_avx2(d, s, n);
    else
        memcpy(d, s, n);
}

// Copying lists into page-locked staging memory.  One thread's memcpy of
// lists just built elsewhere runs at about 15 GB/s on the GPU's host; the
// copy is split between the calling thread and a few persistent workers
// that spin briefly between calls and then sleep (a parallel region per
// call costs more than the copy it splits).
#ifndef GRAV_COPY_WORKERS
#define GRAV_COPY_WORKERS 4
#endif
struct CopyPool {
    static constexpr int kWorkers = GRAV_COPY_WORKERS;
    static constexpr size_t kPart = 64u << 10;  // below this a list is copied by one thread
    std::thread th[kWorkers];
    bool started = false;
    bool retired = false;
    std::atomic<uint64_t> gen{0};
    std::atomic<int> remaining{0};
    std::atomic<int> sleepers{0};
    std::atomic<bool> stop{false};
    std::mutex mu;
    std::condition_variable cv;
    char *dst = nullptr;
    const char *src = nullptr;
    size_t bytes = 0, per = 0;
    int parts = 0;

    void part(int k) {
        const size_t a = (size_t)k * per, b = std::min(bytes, a + per);
        if (a < b)
            copy_bytes(dst + a, src + a, b - a);
    }
    void worker(int w) {
        uint64_t seen = 0;
        while (true) {
            uint64_t g = gen.load(std::memory_order_acquire);
            for (int spin = 0; g == seen && spin < 20000 && !stop.load(); spin++)
                g = gen.load(std::memory_order_acquire);
            if (g == seen) {
                std::unique_lock<std::mutex> lk(mu);
                sleepers++;
                cv.wait_for(lk, std::chrono::milliseconds(20), [&] {
                    return stop.load() || gen.load(std::memory_order_acquire) != seen;
                });
                sleepers--;
                if (stop.load())
                    return;
                continue;
            }
            seen = g;
            if (w + 1 < parts)
                part(w + 1);
            // every worker acknowledges every generation, with or without a
            // part: the caller publishes the next copy only after all have,
            // so no worker can read one copy's generation and another's
            // fields (parts, pointers)
            remaining.fetch_sub(1, std::memory_order_release);
        }
    }
    // 0, or -1 when the workers did not acknowledge within the bound: the
    // copy is then complete (done here) but a late worker may still write
    // into d, so the pool retires (later copies run on the calling thread
    // alone and publish no generation) and the call reports the failure.
    int copy(void *d, const void *sr, size_t n) {
        const int np = (int)std::min<size_t>(kWorkers + 1, n / kPart + 1);
        if (np <= 1 || retired) {
            copy_bytes((char *)d, (const char *)sr, n);
            return 0;
        }
        if (!started) {
            for (int w = 0; w < kWorkers; w++) th[w] = std::thread([this, w] { worker(w); });
            started = true;
            atexit([] { shutdown_pool(); });
        }
        dst = (char *)d;
        src = (const char *)sr;
        bytes = n;
        parts = np;
        per = (n / np + 63) / 64 * 64;
        remaining.store(kWorkers, std::memory_order_relaxed);
        gen.fetch_add(1, std::memory_order_release);
        if (sleepers.load()) {
            std::lock_guard<std::mutex> lk(mu);
            cv.notify_all();
        }
        part(0);
        // the workers' parts and acknowledgements, with a bound
        if (!wait_until([&] { return remaining.load(std::memory_order_acquire) == 0; }, 10.0)) {
            memcpy(d, sr, n);
            retired = true;
            return -1;
        }
        return 0;
    }
    static void shutdown_pool();
};
CopyPool *g_pool = nullptr;

void CopyPool::shutdown_pool() {
    if (!g_pool || !g_pool->started)
        return;
    {
        std::lock_guard<std::mutex> lk(g_pool->mu);
        g_pool->stop.store(true);
    }
    g_pool->cv.notify_all();
    for (auto &t : g_pool->th)
        if (t.joinable())
            t.join();
    g_pool->started = false;
}

int stage_copy(void *dst, const void *src, size_t bytes) {
    if (!g_pool)
        g_pool = new CopyPool();
    if (g_pool->copy(dst, src, bytes))
        return gc::set_status(-1, "staging copy: the copy workers did not finish within 10 s "
                                  "(copies continue on the calling thread)");
    return 0;
}

int check_device_error(const char *what) {
    unsigned h = 0;
    GC_CHECK(cudaMemcpy(&h, S.derr, sizeof(h), cudaMemcpyDeviceToHost));
    if (h) {
        GC_CHECK(cudaMemset(S.derr, 0, sizeof(unsigned)));
        return gc::set_status(-2, "%s: device error word 0x%x (1 wait timeout, 2 bad index, 4 run checksum)",
                              what, h);
    }
    return 0;
}

template <int ORDER, int SOFT>
int launch_list(cudaStream_t st, const float *pos, float4 *acc, int m, const float *f, int nblk,
                int sz, float e, float qsh) {
    constexpr int REC = RecOf<ORDER>::v;
    int threads = min(128, ((m + SPT - 1) / SPT + 31) / 32 * 32);
    int gx = (m + threads * SPT - 1) / (threads * SPT);
    // split the list so that one call spreads over the SMs
    int want = max(1, (2 * S.nsm) / gx);
    int bpc = max(TBLK, (nblk + want - 1) / want);
    bpc = (bpc + TBLK - 1) / TBLK * TBLK;
    int gy = (nblk + bpc - 1) / bpc;
    size_t smem = (size_t)2 * TBLK * sz * 8 * 4 + (size_t)TSRC * REC * 4 + 16;
    auto kern = k_list<ORDER, SOFT>;
    // the largest dynamic shared memory set for this kernel so far (once per size)
    static int smem_set = 0;
    if ((int)smem > smem_set) {
        GC_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        smem_set = (int)smem;
    }
    kern<<<dim3(gx, gy), threads, smem, st>>>(pos, acc, m, f, nblk, sz, bpc, e, qsh, S.derr);
    GC_CHECK(cudaGetLastError());
    return 0;
}

struct Routine {
    const char *name;
    int order, soft, sz_min;
    float qsh;
};
const Routine kRoutines[] = {
    {"pM", 0, SOFT_NONE, 4, 0.f},        {"pQ", 2, SOFT_NONE, 13, -0.5f},
    {"pH", 4, SOFT_NONE, 29, 0.5f},      {"pM_sK1", 0, SOFT_K1, 4, 0.f},
    {"pMp", 0, SOFT_PLUMMER, 4, 0.f},    {"pQp", 2, SOFT_PLUMMER, 13, -0.5f},
    {"pHp", 4, SOFT_PLUMMER, 29, 0.5f},  {"pMs", 0, SOFT_MASKED, 4, 0.f},
};

int dispatch_list(const Routine &r, cudaStream_t st, const float *pos, float4 *acc, int m,
                  const float *f, int nblk, int sz, float e) {
#define GC_CASE(O, SO)                                                        \
    if (r.order == O && r.soft == SO)                                         \
        return launch_list<O, SO>(st, pos, acc, m, f, nblk, sz, e, r.qsh);
    GC_CASE(0, SOFT_NONE)
    GC_CASE(2, SOFT_NONE)
    GC_CASE(4, SOFT_NONE)
    GC_CASE(0, SOFT_K1)
    GC_CASE(0, SOFT_PLUMMER)
    GC_CASE(2, SOFT_PLUMMER)
    GC_CASE(4, SOFT_PLUMMER)
    GC_CASE(0, SOFT_MASKED)
#undef GC_CASE
    return gc::set_status(-1, "no kernel for routine %s", r.name);
}

// ---- deferred issue: the submitter thread ----
// grav_mn_CUDA copies its list into a slot's staging buffer and queues a
// job; one submitter thread takes the jobs in order and issues, on the
// slot's stream, the copy to the device, the event that frees the staging
// buffer, and the launch.  Errors there set the status as in the calling
// thread (abort in the default error mode), and drain_all returns them.
struct Job {
    const Routine *r;
    int q, turn, n, nblk, sz;
    int64_t first;
    size_t bytes;
    float e;
};

struct Submitter {
    static constexpr int kCap = 256;
    Job ring[kCap];
    std::atomic<uint64_t> head{0}, tail{0};  // next job to push / to issue
    std::atomic<bool> sleeping{false}, stop{false};
    std::atomic<int> err{0};
    std::mutex mu;
    std::condition_variable cv;
    std::thread th;
    bool started = false;
    // staging buffers whose copies were issued, oldest first: polled while
    // the queue is empty and marked free when their copy has completed, so
    // the caller rarely waits on an event
    std::pair<int, int> issued[kCap];
    uint64_t issued_head = 0, issued_tail = 0;

    void poll_slots() {
        for (int q = 0; q < NQ; q++) {
            Slot &s = S.q[q];
            if (s.kpending.load(std::memory_order_acquire) == 1 &&
                s.queued.load(std::memory_order_acquire) == 0 &&
                cudaEventQuery(s.kdone) == cudaSuccess)
                s.kpending.store(0, std::memory_order_release);
        }
    }
    void poll_issued() {
        while (issued_tail != issued_head) {
            const auto [q, k] = issued[issued_tail % kCap];
            Slot &s = S.q[q];
            if (s.bstate[k].load(std::memory_order_acquire) != 2) {  // taken over by the caller
                issued_tail++;
                continue;
            }
            if (cudaEventQuery(s.copied[k]) != cudaSuccess)
                return;
            int two = 2;
            s.bstate[k].compare_exchange_strong(two, 0, std::memory_order_acq_rel);
            issued_tail++;
        }
    }

    void issue(const Job &j) {
        const int64_t t0 = now_ns();
        Slot &s = S.q[j.q];
        cudaError_t e = cudaMemcpyAsync(s.dev, s.hbuf[j.turn], j.bytes, cudaMemcpyHostToDevice,
                                        s.stream);
        if (e == cudaSuccess)
            e = cudaEventRecord(s.copied[j.turn], s.stream);
        s.bstate[j.turn].store(2, std::memory_order_release);
        if (issued_head - issued_tail < (uint64_t)kCap)
            issued[issued_head++ % kCap] = {j.q, j.turn};
        int rc = e == cudaSuccess ? 0 : gc::cuda_status(e, "grav_mn_CUDA: list copy");
        if (!rc)
            rc = dispatch_list(*j.r, s.stream, S.devpos + 3 * j.first, S.devaccp + j.first, j.n,
                               (const float *)s.dev, j.nblk, j.sz, j.e);
        if (!rc && cudaEventRecord(s.kdone, s.stream) == cudaSuccess)
            s.kpending.store(1, std::memory_order_release);
        if (rc) {
            int zero = 0;
            err.compare_exchange_strong(zero, rc);
        }
        g_phase_ns[3] += now_ns() - t0;
        s.queued.fetch_sub(1, std::memory_order_release);
    }
    void run() {
        while (true) {
            const uint64_t t = tail.load(std::memory_order_relaxed);
            if (t == head.load(std::memory_order_acquire)) {
                poll_issued();
                poll_slots();
                bool got = false;
                for (int spin = 0; spin < 20000 && !got; spin++)
                    got = t != head.load(std::memory_order_acquire);
                if (!got) {
                    std::unique_lock<std::mutex> lk(mu);
                    sleeping.store(true);
                    cv.wait_for(lk, std::chrono::milliseconds(50), [&] {
                        return stop.load() || t != head.load(std::memory_order_acquire);
                    });
                    sleeping.store(false);
                }
                if (stop.load() && t == head.load(std::memory_order_acquire))
                    return;
                continue;
            }
            issue(ring[t % kCap]);
            tail.store(t + 1, std::memory_order_release);
        }
    }
    int push(const Job &j) {
        if (!started) {
            th = std::thread([this] { run(); });
            started = true;
            atexit([] { shutdown_submitter(); });
        }
        const uint64_t h = head.load(std::memory_order_relaxed);
        const int64_t t0 = now_ns();
        if (!wait_until([&] { return h - tail.load(std::memory_order_acquire) < (uint64_t)kCap; }))
            return gc::set_status(-1, "grav_mn_CUDA: the submitter stopped taking jobs");
        g_phase_ns[2] += now_ns() - t0;
        ring[h % kCap] = j;
        S.q[j.q].queued.fetch_add(1, std::memory_order_release);
        head.store(h + 1, std::memory_order_release);
        if (sleeping.load()) {
            std::lock_guard<std::mutex> lk(mu);
            cv.notify_one();
        }
        return 0;
    }
    int drain() {
        const int64_t t0 = now_ns();
        struct Add {
            int64_t t0;
            ~Add() { g_phase_ns[4] += now_ns() - t0; }
        } add{t0};
        if (!wait_until([&] {
                return tail.load(std::memory_order_acquire) == head.load(std::memory_order_acquire);
            }))
            return gc::set_status(-1, "grav_mn_CUDA: the submitter did not drain");
        return err.exchange(0);
    }
    static void shutdown_submitter();
};
Submitter *g_sub = nullptr;

void Submitter::shutdown_submitter() {
    if (!g_sub || !g_sub->started)
        return;
    g_sub->drain();
    {
        std::lock_guard<std::mutex> lk(g_sub->mu);
        g_sub->stop.store(true);
    }
    g_sub->cv.notify_one();
    if (g_sub->th.joinable())
        g_sub->th.join();
    g_sub->started = false;
}

Submitter &submitter() {
    if (!g_sub)
        g_sub = new Submitter();
    return *g_sub;
}

int grav_mn_impl(const char *routine, const float *p, int n, int stride, const float *f,
                 int source_n, int sz, float e, int q) {
    std::lock_guard<std::recursive_mutex> call_lock(g_call_mu);
    if (ensure_init())
        return gc::g_status;
    const Routine *r = nullptr;
    for (const Routine &c : kRoutines)
        if (routine && strcmp(routine, c.name) == 0)
            r = &c;
    if (!r)
        return gc::set_status(-1, "routine %s not found", routine ? routine : "(null)");
    if (!S.devpos || !S.Btab)
        return gc::set_status(-1, "grav_mn_CUDA before WalkInitSinkCUDA");
    if (stride != S.bstride)
        return gc::set_status(-1, "stride %d differs from the registered %d", stride, S.bstride);
    if (sz < r->sz_min || source_n < 0 || source_n % 8 || n < 0)
        return gc::set_status(-1, "bad list shape: sz %d source_n %d n %d for %s", sz, source_n, n,
                              routine);
    int64_t first = (p - S.Btab) / stride;
    if (first < 0 || first + n > S.nobj)
        return gc::set_status(-1, "sinks [%lld, %lld) outside the registered %lld",
                              (long long)first, (long long)(first + n), (long long)S.nobj);
    if (n == 0 || source_n == 0)
        return 0;
    size_t bytes = (size_t)source_n * sz * sizeof(float);
    if (int rc = slot_reserve(q, bytes))
        return rc;
    Slot &s = S.q[q];
    const int64_t t0 = now_ns();
    const int copied = stage_copy(s.host, f, bytes);
    g_phase_ns[0] += now_ns() - t0;
    if (copied)
        return copied;
    g_phase_calls++;
    s.bstate[s.turn].store(1, std::memory_order_release);
    s.inuse = true;
    return submitter().push(Job{r, q, s.turn, n, source_n / 8, sz, first, bytes, e});
}

}  // namespace

// ------------------------------------------------------------ entry points
extern "C" void CUDA_Init(void *device_prop) {
    (void)device_prop;
    if (ensure_init())
        return;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, 0) == cudaSuccess && getenv("GRAVCUDA_VERBOSE"))
        fprintf(stderr, "CUDA_Init: %s, sm_%d%d, %d SMs, %.1f GB\n", prop.name, prop.major,
                prop.minor, prop.multiProcessorCount, prop.totalGlobalMem / 1e9);
}

extern "C" void CUDA_Finalize(void) {
    std::lock_guard<std::recursive_mutex> call_lock(g_call_mu);
    grav_groups_release_CUDA();
    Submitter::shutdown_submitter();
    if (!S.init)
        return;
    for (int i = 0; i < NQ; i++) {
        Slot &s = S.q[i];
        if (s.stream) {
            cudaStreamSynchronize(s.stream);
            cudaStreamDestroy(s.stream);
        }
        for (int k = 0; k < 2; k++) {
            if (s.hbuf[k])
                cudaFreeHost(s.hbuf[k]);
            if (s.copied[k])
                cudaEventDestroy(s.copied[k]);
        }
        if (s.kdone)
            cudaEventDestroy(s.kdone);
        if (s.dev)
            cudaFree(s.dev);
        s.reset();
    }
    cudaFree(S.devpos);
    cudaFree(S.devaccp);
    cudaFree(S.qdev);
    cudaFree(S.derr);
    S.init = false;
    S.Btab = nullptr;
    S.bstride = 0;
    S.nobj = 0;
    S.devpos = nullptr;
    S.devaccp = nullptr;
    S.qdev = nullptr;
    S.ncells = 0;
    S.derr = nullptr;
}

extern "C" int vecwidthCUDA(void) { return SPT; }

extern "C" void gravcuda_dropin_phases(double out[6]) {
    for (int k = 0; k < 5; k++) out[k] = 1e-9 * (double)g_phase_ns[k].load();
    out[5] = (double)g_phase_calls.load();
}

extern "C" int qallocCUDA(int *inuse) {
    std::lock_guard<std::recursive_mutex> call_lock(g_call_mu);
    if (ensure_init())
        return -1;
    // slots are handed out round-robin; without the busy count the search
    // stops at the first free slot (one stream query per busy slot passed)
    static int next = 0;
    int busy = 0, free_slot = -1;
    for (int k = 0; k < NQ; k++) {
        const int i = (next + k) % NQ;
        Slot &s = S.q[i];
        if (s.inuse && s.queued.load(std::memory_order_acquire) == 0 &&
            s.kpending.load(std::memory_order_acquire) == 0 && g_sub && g_sub->started)
            s.inuse = false;  // the submitter saw its last launch complete
        if (s.inuse && s.queued.load(std::memory_order_acquire) == 0) {
            cudaError_t e = cudaStreamQuery(s.stream);
            if (e == cudaSuccess) {
                s.inuse = false;
                s.kpending.store(0, std::memory_order_release);
            } else if (e != cudaErrorNotReady) {
                gc::cuda_status(e, "cudaStreamQuery");
                return -1;
            }
        }
        if (s.inuse)
            busy++;
        else if (free_slot < 0) {
            free_slot = i;
            if (!inuse)
                break;
        }
    }
    if (inuse)
        *inuse = busy;
    if (free_slot >= 0)
        next = (free_slot + 1) % NQ;
    return free_slot;
}

extern "C" void WalkInitSrcCUDA(float *qtab, int stride, int64_t nobj) {
    std::lock_guard<std::recursive_mutex> call_lock(g_call_mu);
    if (ensure_init())
        return;
    if (!qtab || stride < 20 || nobj <= 0) {
        gc::set_status(-1, "WalkInitSrcCUDA: bad table (stride %d floats, need >= 20)", stride);
        return;
    }
    std::vector<float> h((size_t)nobj * 13);
    for (int64_t i = 0; i < nobj; i++) {
        const float *c = qtab + (size_t)i * stride;
        float *o = &h[(size_t)i * 13];
        o[0] = c[0];                                  // mass
        o[1] = c[1]; o[2] = c[2]; o[3] = c[3];        // pos
        o[4] = c[5];                                  // bmax
        for (int k = 0; k < 5; k++) o[5 + k] = c[15 + k];  // qxx qxy qyy qxz qyz
        for (int k = 0; k < 3; k++) o[10 + k] = c[12 + k];  // qx qy qz
    }
    cudaFree(S.qdev);
    S.qdev = nullptr;
    if (cudaMalloc(&S.qdev, h.size() * 4) != cudaSuccess ||
        cudaMemcpy(S.qdev, h.data(), h.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
        gc::set_status(-1, "WalkInitSrcCUDA: device copy failed");
        return;
    }
    S.ncells = nobj;
}

extern "C" void WalkTerminateSrcCUDA(void) {
    std::lock_guard<std::recursive_mutex> call_lock(g_call_mu);
    if (S.qdev)
        cudaFree(S.qdev);
    S.qdev = nullptr;
    S.ncells = 0;
}

static int drain_all();

extern "C" void WalkInitSinkCUDA(float *btab, int stride, int64_t nobj) {
    std::lock_guard<std::recursive_mutex> call_lock(g_call_mu);
    if (ensure_init())
        return;
    if (drain_all())  // queued lists of an earlier walk still read the old tables
        return;
    for (auto &x : g_phase_ns) x = 0;
    g_phase_calls = 0;
    if (!btab || stride < 4 || nobj <= 0) {
        gc::set_status(-1, "WalkInitSinkCUDA: bad table");
        return;
    }
    cudaFree(S.devpos);
    cudaFree(S.devaccp);
    S.devpos = nullptr;
    S.devaccp = nullptr;
    std::vector<float> h((size_t)nobj * 3);
    for (int64_t i = 0; i < nobj; i++)
        for (int d = 0; d < 3; d++) h[3 * i + d] = btab[(size_t)i * stride + 1 + d];
    if (cudaMalloc(&S.devpos, h.size() * 4) != cudaSuccess ||
        cudaMalloc(&S.devaccp, (size_t)nobj * sizeof(float4)) != cudaSuccess ||
        cudaMemcpy(S.devpos, h.data(), h.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(S.devaccp, 0, (size_t)nobj * sizeof(float4)) != cudaSuccess) {
        gc::set_status(-1, "WalkInitSinkCUDA: device allocation failed");
        return;
    }
    S.Btab = btab;
    S.bstride = stride;
    S.nobj = nobj;
}

static int drain_all() {
    if (g_sub && g_sub->started)
        if (int rc = g_sub->drain())
            return rc;
    for (int i = 0; i < NQ; i++) {
        if (S.q[i].stream)
            GC_CHECK(cudaStreamSynchronize(S.q[i].stream));
        S.q[i].inuse = false;
    }
    return 0;
}

extern "C" int gravcuda_peek_accumulators(float *out, int64_t first, int64_t count) {
    std::lock_guard<std::recursive_mutex> call_lock(g_call_mu);
    if (!S.devaccp || first < 0 || first + count > S.nobj)
        return gc::set_status(-1, "gravcuda_peek_accumulators: range outside the sink table");
    if (int rc = drain_all())
        return rc;
    GC_CHECK(cudaMemcpy(out, S.devaccp + first, count * sizeof(float4), cudaMemcpyDeviceToHost));
    return check_device_error("list kernels");
}

extern "C" void WalkTerminateSinkCUDA(float *btab, int stride, int64_t nobj) {
    std::lock_guard<std::recursive_mutex> call_lock(g_call_mu);
    if (!S.devaccp) {
        gc::set_status(-1, "WalkTerminateSinkCUDA before WalkInitSinkCUDA");
        return;
    }
    if (nobj != S.nobj || stride < 11) {
        gc::set_status(-1, "WalkTerminateSinkCUDA: table differs from WalkInitSinkCUDA");
        return;
    }
    std::vector<float> h((size_t)nobj * 4);
    if (gravcuda_peek_accumulators(h.data(), 0, nobj))
        return;
    for (int64_t i = 0; i < nobj; i++)
        for (int k = 0; k < 4; k++) btab[(size_t)i * stride + 7 + k] += h[4 * i + k];
    cudaFree(S.devpos);
    cudaFree(S.devaccp);
    S.devpos = nullptr;
    S.devaccp = nullptr;
    S.Btab = nullptr;
    S.nobj = 0;
}

extern "C" int grav_mn_status_CUDA(const char *routine, const float *p, const int n,
                                   const int stride, const float *f, const int source_n,
                                   const int sz, const float e, int q) {
    return grav_mn_impl(routine, p, n, stride, f, source_n, sz, e, q);
}

extern "C" void grav_mn_CUDA(const char *routine, const float *p, float *accp, const int n,
                             const int stride, const float *f, const int source_n, const int sz,
                             const float e, int *ncut, int q) {
    (void)accp;
    (void)ncut;
    grav_mn_impl(routine, p, n, stride, f, source_n, sz, e, q);
}

static int runs_launch(int sink_base, int m, const uint16_t *ss_index, const segment *ss_seg,
                       int ss_len, const segment *seg, int seg_len, int source_base,
                       const int *source_n, float mmass, float e, int q) {
    std::lock_guard<std::recursive_mutex> call_lock(g_call_mu);
    if (ensure_init())
        return gc::g_status;
    if (!S.devpos)
        return gc::set_status(-1, "body-run kernel before WalkInitSinkCUDA");
    if (sink_base < 0 || m < 0 || sink_base + (int64_t)m > S.nobj || source_base < 0 ||
        source_base > S.nobj)
        return gc::set_status(-1, "body-run kernel: sinks or sources outside the table");
    if (m == 0)
        return 0;
    // one device buffer: group_of | group runs | expected counts | runs (128-byte aligned parts)
    auto al = [](size_t x) { return (x + 127) & ~(size_t)127; };
    size_t o_idx = 0, n_idx = ss_index ? (size_t)m * 2 : 0;
    size_t o_gs = al(o_idx + n_idx), n_gs = (size_t)ss_len * sizeof(segment);
    size_t o_cnt = al(o_gs + n_gs), n_cnt = source_n ? (size_t)ss_len * 4 : 0;
    size_t o_seg = al(o_cnt + n_cnt), n_seg = (size_t)seg_len * sizeof(segment);
    size_t total = o_seg + n_seg;
    if (int rc = slot_quiet(q))
        return rc;
    if (int rc = slot_reserve(q, total))
        return rc;
    Slot &s = S.q[q];
    char *h = (char *)s.host, *d = (char *)s.dev;
    if (n_idx)
        memcpy(h + o_idx, ss_index, n_idx);
    memcpy(h + o_gs, ss_seg, n_gs);
    if (n_cnt)
        memcpy(h + o_cnt, source_n, n_cnt);
    memcpy(h + o_seg, seg, n_seg);
    for (int i = 0; ss_index && i < m; i++)
        if (ss_index[i] >= ss_len)
            return gc::set_status(-1, "ss_index[%d] = %d >= ss_len %d", i, ss_index[i], ss_len);
    GC_CHECK(cudaMemcpyAsync(d, h, total, cudaMemcpyHostToDevice, s.stream));
    if (int rc = slot_copied(s))
        return rc;
    s.inuse = true;
    s.kpending.store(2, std::memory_order_release);  // launched here: query the stream
    int threads = 128;
    k_runs_k1<<<(m + threads - 1) / threads, threads, 0, s.stream>>>(
        S.devpos + 3 * (size_t)sink_base, S.devaccp + sink_base, m,
        ss_index ? (const uint16_t *)(d + o_idx) : nullptr, (const segment *)(d + o_gs),
        (const segment *)(d + o_seg), seg_len, S.devpos + 3 * (size_t)source_base,
        (int)(S.nobj - source_base), n_cnt ? (const int *)(d + o_cnt) : nullptr, mmass, e,
        S.derr);
    GC_CHECK(cudaGetLastError());
    return 0;
}

extern "C" void grav_mns_CUDA(const char *routine, const int base, const int m,
                              const segment *seg, const int seg_n, const int source_n,
                              const float mmass, float e, int *ncut, int q) {
    (void)ncut;
    if (!routine || strcmp(routine, "pMM_sK1") != 0) {
        gc::set_status(-1, "routine %s not found", routine ? routine : "(null)");
        return;
    }
    segment whole{0u, (unsigned)seg_n};
    runs_launch(base, m, nullptr, &whole, 1, seg, seg_n, 0, &source_n, mmass, e, q);
}

extern "C" void grav_mnss_CUDA(const char *routine, const int sink_base, const int m,
                               const uint16_t *ss_index, const segment *ss_seg, const int ss_len,
                               const segment *seg, const int seg_len, const int source_base,
                               const int *source_n, const float mmass, float e, int *ncut,
                               int q) {
    (void)ncut;
    if (!routine || strcmp(routine, "pMM_mnss_sK1") != 0) {
        gc::set_status(-1, "routine %s not found", routine ? routine : "(null)");
        return;
    }
    runs_launch(sink_base, m, ss_index, ss_seg, ss_len, seg, seg_len, source_base, source_n,
                mmass, e, q);
}

extern "C" void grav_qns_CUDA(const char *routine, const int base, const int m,
                              const int *source_list, const int source_n, int q) {
    std::lock_guard<std::recursive_mutex> call_lock(g_call_mu);
    if (ensure_init())
        return;
    if (!routine || strcmp(routine, "pQQ1") != 0) {
        gc::set_status(-1, "routine %s not found", routine ? routine : "(null)");
        return;
    }
    if (!S.qdev || !S.devpos) {
        gc::set_status(-1, "grav_qns_CUDA needs WalkInitSrcCUDA and WalkInitSinkCUDA");
        return;
    }
    if (base < 0 || m < 0 || base + (int64_t)m > S.nobj || source_n < 0) {
        gc::set_status(-1, "grav_qns_CUDA: sinks outside the table");
        return;
    }
    if (m == 0 || source_n == 0)
        return;
    size_t bytes = (size_t)source_n * sizeof(int);
    if (slot_quiet(q) || slot_reserve(q, bytes))
        return;
    Slot &s = S.q[q];
    memcpy(s.host, source_list, bytes);
    if (cudaMemcpyAsync(s.dev, s.host, bytes, cudaMemcpyHostToDevice, s.stream) != cudaSuccess) {
        gc::set_status(-1, "grav_qns_CUDA: copy failed");
        return;
    }
    if (slot_copied(s))
        return;
    s.inuse = true;
    s.kpending.store(2, std::memory_order_release);  // launched here: query the stream
    k_quad_index<<<(m + 127) / 128, 128, 0, s.stream>>>(S.devpos + 3 * (size_t)base,
                                                        S.devaccp + base, m, (const int *)s.dev,
                                                        source_n, S.qdev, (int)S.ncells, S.derr);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess)
        gc::cuda_status(err, "k_quad_index");
}

extern "C" void grav_qnss_CUDA(const char *routine, const int base, const int m,
                               const segment *seg, const float *source, const int source_n,
                               int q) {
    std::lock_guard<std::recursive_mutex> call_lock(g_call_mu);
    if (ensure_init())
        return;
    if (!routine || strcmp(routine, "pQ1_qnss") != 0) {
        gc::set_status(-1, "routine %s not found", routine ? routine : "(null)");
        return;
    }
    if (!S.devpos || base < 0 || m < 0 || base + (int64_t)m > S.nobj || source_n % 8) {
        gc::set_status(-1, "grav_qnss_CUDA: bad sinks or source_n %d", source_n);
        return;
    }
    if (m == 0)
        return;
    auto al = [](size_t x) { return (x + 127) & ~(size_t)127; };
    size_t n_seg = (size_t)m * sizeof(segment);
    size_t o_src = al(n_seg), n_src = (size_t)source_n * 13 * sizeof(float);
    if (slot_quiet(q) || slot_reserve(q, o_src + n_src))
        return;
    Slot &s = S.q[q];
    memcpy(s.host, seg, n_seg);
    memcpy((char *)s.host + o_src, source, n_src);
    if (cudaMemcpyAsync(s.dev, s.host, o_src + n_src, cudaMemcpyHostToDevice, s.stream) !=
        cudaSuccess) {
        gc::set_status(-1, "grav_qnss_CUDA: copy failed");
        return;
    }
    if (slot_copied(s))
        return;
    s.inuse = true;
    s.kpending.store(2, std::memory_order_release);  // launched here: query the stream
    k_quad_runs<<<(m + 127) / 128, 128, 0, s.stream>>>(
        S.devpos + 3 * (size_t)base, S.devaccp + base, m, (const segment *)s.dev,
        (const float *)((char *)s.dev + o_src), source_n, S.derr);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess)
        gc::cuda_status(err, "k_quad_runs");
}
