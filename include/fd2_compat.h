/*
 * fd2_compat.h -- Fortran-callable drop-ins for hybridMANTIS's penEasy side.
 *
 * gpuoptical_ and cpuoptical_ keep the reference's names, by-reference
 * arguments and data exchange through the Fortran COMMON blocks, so the
 * EDE tally (main/hybridMANTIS_tallyEnergyDepositionEvents.f:257-313) and
 * the main program's final flush (main/hybridMANTIS_penEasy.f:436-443)
 * link against libfd2.so unchanged.  The COMMON blocks are defined by the
 * Fortran program; the library references them weakly and reports
 * FD2_ERR_STATE through fd2_compat_status() when they are absent.
 *
 *   gpuoptical_(penctr, myfactGPU)   main/hybridMANTIS_cuda_ver1_0.cu:107
 *     99  create the GPU context from /inputargs/ (cuda:187-228)
 *     100 wait for the previous buffer, transport optical_ events
 *         [0, *myfactGPU) asynchronously (cuda:229-279)
 *     101 the same for the last buffer, then wait, add the PRF into
 *         /outputimage/, bin the per-history counts into /outputdetprim/,
 *         add the counters into /optstats/ and release the context
 *         (cuda:287-446)
 *   cpuoptical_(gpusize)             main/hybridMANTIS_c_ver1_0.c:81
 *     transports optical_ events [*gpusize, myctropt) synchronously -- on
 *     the GPU: there is no CPU transport in this library -- and adds its
 *     PRF, PHS and counters into the COMMON blocks before returning, as
 *     the reference's CPU path does per call (c:342-372).
 *   gpuoptlb_(gptime, lbbuf)         main/hybridMANTIS_cuda_ver1_0_LB.cu:108
 *   cpuoptlb_(cptime, cpubufsize)    main/hybridMANTIS_c_ver1_0_LB.c:86
 *     load-balancing probes (tally.f:198-210): transport optical_ events
 *     [0, *lbbuf) (resp. [0, *cpubufsize)) synchronously -- both on the
 *     GPU -- add the results into the COMMON blocks and return the elapsed
 *     seconds in *gptime (resp. *cptime).
 */
#ifndef FD2_COMPAT_H
#define FD2_COMPAT_H

#include "fd2.h"

#ifdef __cplusplus
extern "C" {
#endif

#define FD2_GPUBUFSIZE 2304000 /* gpubufsize = maxvalopt, cuda:62 */

/* Layouts of the Fortran COMMON blocks (kernel_cuda_c_ver1_0.cu:84-236). */
struct fd2_common_optical {
    double xbufopt[FD2_GPUBUFSIZE]; /* cm */
    double ybufopt[FD2_GPUBUFSIZE];
    double zbufopt[FD2_GPUBUFSIZE];
    double debufopt[FD2_GPUBUFSIZE]; /* eV */
    int nbufopt[FD2_GPUBUFSIZE];     /* 1-based history */
    int myctropt;
    int cpu_num_real;
};
struct fd2_common_inputargs {
    double detx, dety, detheight, detradius, detnC, detnIC, dettop, detbulk, detbeta;
    double detdmin, detdmax, detlboundx, detlboundy, detuboundx, detuboundy, detyield, detsensorRefl;
    int detpixel, rungpu, machinenum, mynumhist, minphotons, maxphotons, mynumbins;
};
struct fd2_common_optstats {
    double glgen, gldetect, glabstop, glabsbulk, gllost, gloutofcol, gltheta1, glgputime;
};
struct fd2_common_outputdetprim {
    int gldetprimary[1000];
};
struct fd2_common_outputimage {
    unsigned long long newimageopt[501][501];
    unsigned long long tempimageopt[501][501];
};

FD2_API void gpuoptical_(int *penctr, int *myfactGPU);
FD2_API void cpuoptical_(int *gpusize);
FD2_API void gpuoptlb_(double *gptime, int *lbbuf);
FD2_API void cpuoptlb_(double *cptime, int *cpubufsize);

/* Status of the last shim call (the shims return void, as the reference's). */
FD2_API fd2_status fd2_compat_status(void);

#ifdef __cplusplus
}
#endif
#endif
