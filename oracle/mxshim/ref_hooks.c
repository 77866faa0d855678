/*
 * ref_hooks.c — link-time hooks compiled into each oracle/_ref library.
 *
 * TEST INFRASTRUCTURE ONLY. The reference seeds its CPU RNG from the monotonic
 * clock (+MCmatlab/src/MCmatlab.c:241 via getMicroSeconds, MCmatlablib.c:202-211)
 * and sizes its OpenMP team from omp_get_num_procs() (MCmatlab.c:728,
 * finiteElementHeatPropagator.c:756). The libraries are linked with
 * -Wl,--wrap=clock_gettime,--wrap=omp_get_num_procs so a harness can pin the seed
 * (mxshim_fixed_us >= 0) and the thread count (mxshim_nprocs > 0); with both left
 * at their defaults the reference runs exactly as built.
 */
#define _GNU_SOURCE
#include <time.h>

extern long long mxshim_fixed_us;
extern int mxshim_nprocs;

int __real_clock_gettime(clockid_t clk, struct timespec *ts);
int __wrap_clock_gettime(clockid_t clk, struct timespec *ts) {
  if (mxshim_fixed_us >= 0) {
    ts->tv_sec = (time_t)(mxshim_fixed_us / 1000000);
    ts->tv_nsec = (long)(mxshim_fixed_us % 1000000) * 1000;
    return 0;
  }
  return __real_clock_gettime(clk, ts);
}

#ifdef _OPENMP
int __real_omp_get_num_procs(void);
int __wrap_omp_get_num_procs(void) {
  return mxshim_nprocs > 0 ? mxshim_nprocs : __real_omp_get_num_procs();
}
#endif
