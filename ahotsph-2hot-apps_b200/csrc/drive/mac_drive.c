/*
 * mac_drive.c -- a caller of the drop-in ABI the way nln/mac.c drives it,
 * for timing the drop-in path without an interpreter in the loop.
 *
 * For every sink group and list kind (nln/mac.c:1212-1218: one grav_mn_CUDA
 * per node and kind, on a slot from qallocCUDA, polled while none is free,
 * nln/mac.c:964-971) the group's reference AoSoA list is handed to
 * grav_mn_CUDA, then WalkTerminateSinkCUDA waits for all of them and adds
 * the results into the body table (nln/mac.c:257-277).  WalkInitSinkCUDA is
 * the caller's (once per step, outside the timing).
 */
#include <stdint.h>
#include <time.h>

#include "gravcuda.h"

static double now_s(void) {
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

/*
 * btab: the body table registered by WalkInitSinkCUDA (stride floats per
 * body, nobj bodies); group g owns sinks [first[g], first[g] + count[g]).
 * For list kind k < nkinds: routine[k], record size sz[k] floats, blocks
 * data[k] + blk_ptr[k][g] * sz[k] * 8 .. blk_ptr[k][g + 1] (8 lanes each).
 * e: the routine's softening argument.  Returns the wall-clock seconds from
 * the first call to the end of WalkTerminateSinkCUDA, or -1 on an error
 * (gravcuda_status() says which).
 */
double mac_drive_mn(float *btab, int stride, int64_t nobj, int64_t ngroups, const int64_t *first,
                    const int32_t *count, int nkinds, const char *const *routine, const int *sz,
                    const float *const *data, const int64_t *const *blk_ptr, float e) {
    const double t0 = now_s();
    for (int64_t g = 0; g < ngroups; g++) {
        for (int k = 0; k < nkinds; k++) {
            const int64_t b0 = blk_ptr[k][g], b1 = blk_ptr[k][g + 1];
            if (b1 <= b0)
                continue;
            int q;
            while ((q = qallocCUDA(NULL)) < 0)
                if (gravcuda_status())
                    return -1.0;
            grav_mn_CUDA(routine[k], btab + first[g] * stride, NULL, count[g], stride,
                         data[k] + b0 * sz[k] * 8, (int)(b1 - b0) * 8, sz[k], e, NULL, q);
            if (gravcuda_status())
                return -1.0;
        }
    }
    WalkTerminateSinkCUDA(btab, stride, nobj);
    if (gravcuda_status())
        return -1.0;
    return now_s() - t0;
}
