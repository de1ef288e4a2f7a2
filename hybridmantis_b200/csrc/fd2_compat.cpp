// fd2_compat.cpp -- gpuoptical_ / cpuoptical_ over the C ABI, with the
// reference's Fortran COMMON-block data exchange (see include/fd2_compat.h).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <vector>

#include "fd2.h"
#include "fd2_compat.h"

extern "C" {
// Defined by the Fortran program (or a test driver standing in for it).
extern struct fd2_common_optical optical_ __attribute__((weak));
extern struct fd2_common_inputargs inputargs_ __attribute__((weak));
extern struct fd2_common_optstats optstats_ __attribute__((weak));
extern struct fd2_common_outputdetprim outputdetprim_ __attribute__((weak));
extern struct fd2_common_outputimage outputimage_ __attribute__((weak));
}

namespace {

fd2_status g_status = FD2_OK;
fd2_ctx *g_gpu = nullptr;  // context of the gpuoptical_ path, mode 99 -> 101

bool commons_present()
{
    return &optical_ != nullptr && &inputargs_ != nullptr && &optstats_ != nullptr && &outputdetprim_ != nullptr &&
           &outputimage_ != nullptr;
}

fd2_params params_from_common()
{
    const fd2_common_inputargs &a = inputargs_;
    fd2_params p;
    std::memset(&p, 0, sizeof p);
    p.num_hist = a.mynumhist;
    p.min_photons = a.minphotons;
    p.max_photons = a.maxphotons;
    p.num_bins = a.mynumbins;
    p.det_x = a.detx;
    p.det_y = a.dety;
    p.det_height = a.detheight;
    p.radius = a.detradius;
    p.n_col = a.detnC;
    p.n_gap = a.detnIC;
    p.top_absfrac = a.dettop;
    p.bulk_abs = a.detbulk;
    p.beta = a.detbeta;
    p.d_min = a.detdmin;
    p.d_max = a.detdmax;
    p.lb_x = a.detlboundx;
    p.lb_y = a.detlboundy;
    p.ub_x = a.detuboundx;
    p.ub_y = a.detuboundy;
    p.yield = a.detyield;
    p.pixel = a.detpixel;
    p.sensor_refl = a.detsensorRefl;
    p.run_gpu = a.rungpu;
    p.machine = a.machinenum;
    return p;
}

void report(fd2_status s, fd2_ctx *c, const char *where)
{
    g_status = s;
    if (s != FD2_OK)
        std::fprintf(stderr, "fd2: %s: %s (%s)\n", where, fd2_status_string(s), c ? fd2_last_error(c) : "");
}

fd2_status submit_range(fd2_ctx *c, int from, int to)
{
    const int n = std::max(0, to - from);
    return fd2_submit_events(c, optical_.xbufopt + from, optical_.ybufopt + from, optical_.zbufopt + from,
                             optical_.debufopt + from, optical_.nbufopt + from, n);
}

// Add the context's results into the COMMON blocks (cuda:371-430).
fd2_status accumulate_into_commons(fd2_ctx *c)
{
    fd2_status s;
    int32_t xd = 0, yd = 0;
    if ((s = fd2_get_prf_dims(c, 0, &xd, &yd)) != FD2_OK) return s;
    std::vector<uint64_t> img((size_t)xd * yd);
    if ((s = fd2_get_prf(c, 0, img.data(), (int64_t)img.size())) != FD2_OK) return s;
    for (int ii = 0; ii < std::min(xd, 501); ++ii)
        for (int jj = 0; jj < std::min(yd, 501); ++jj) outputimage_.newimageopt[ii][jj] += img[(size_t)ii * yd + jj];
    const int nb = inputargs_.mynumbins;
    if (nb > 0 && nb <= 1000) {
        std::vector<int32_t> phs((size_t)nb);
        if ((s = fd2_get_phs(c, 0, phs.data(), nb)) != FD2_OK) return s;
        for (int k = 0; k < nb; ++k) outputdetprim_.gldetprimary[k] += phs[(size_t)k];
    }
    fd2_counters k;
    if ((s = fd2_get_counters(c, 0, &k)) != FD2_OK) return s;
    optstats_.glgen += (double)k.generated;
    optstats_.gldetect += (double)k.detected;
    optstats_.glabstop += (double)k.abs_top;
    optstats_.glabsbulk += (double)k.abs_bulk;
    optstats_.gllost += (double)k.lost;
    optstats_.gloutofcol += (double)k.outofcol;
    optstats_.gltheta1 += (double)k.theta1;
    fd2_timing t;
    if (fd2_get_timing(c, &t) == FD2_OK) optstats_.glgputime += (double)t.pipeline_ms;
    return FD2_OK;
}

}  // namespace

extern "C" {

fd2_status fd2_compat_status(void) { return g_status; }

void gpuoptical_(int *penctr, int *myfactGPU)
{
    if (!penctr || !myfactGPU || !commons_present()) return report(FD2_ERR_STATE, nullptr, "gpuoptical_");
    fd2_status s = FD2_OK;
    if (*penctr == 99) {
        if (g_gpu) fd2_destroy(g_gpu);
        g_gpu = nullptr;
        const fd2_params p = params_from_common();
        s = fd2_create(&p, nullptr, &g_gpu);
        return report(s, g_gpu, "gpuoptical_(99)");
    }
    if (!g_gpu) return report(FD2_ERR_STATE, nullptr, "gpuoptical_ before mode 99");
    if (*penctr != 100 && *penctr != 101) return report(FD2_ERR_INVALID_ARGUMENT, g_gpu, "gpuoptical_ mode");
    const int n = std::min(*myfactGPU, FD2_GPUBUFSIZE);
    if ((s = fd2_wait(g_gpu)) == FD2_OK && (s = submit_range(g_gpu, 0, n)) == FD2_OK) s = fd2_run(g_gpu);
    if (s == FD2_OK && *penctr == 101) {
        s = fd2_wait(g_gpu);
        if (s == FD2_OK) s = accumulate_into_commons(g_gpu);
        fd2_destroy(g_gpu);
        g_gpu = nullptr;
    }
    report(s, g_gpu, "gpuoptical_");
}

// Load-balancing probes of the _LB build: transport optical_ events
// [0, *count) synchronously, add the results into the COMMON blocks and
// return the seconds taken (gpuoptlb_, cuda_LB:108-280; cpuoptlb_,
// c_LB:86-286).  Both run on the GPU.
static void lb_probe(double *seconds, int *count, const char *where)
{
    if (!seconds || !count || !commons_present()) return report(FD2_ERR_STATE, nullptr, where);
    const fd2_params p = params_from_common();
    fd2_ctx *c = nullptr;
    fd2_status s = fd2_create(&p, nullptr, &c);
    const auto t0 = std::chrono::steady_clock::now();
    if (s == FD2_OK) s = submit_range(c, 0, std::min(*count, FD2_GPUBUFSIZE));
    if (s == FD2_OK) s = fd2_run(c);
    if (s == FD2_OK) s = fd2_wait(c);
    if (s == FD2_OK) s = accumulate_into_commons(c);
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    report(s, c, where);
    fd2_destroy(c);
}

void gpuoptlb_(double *gptime, int *lbbuf) { lb_probe(gptime, lbbuf, "gpuoptlb_"); }

void cpuoptlb_(double *cptime, int *cpubufsize) { lb_probe(cptime, cpubufsize, "cpuoptlb_"); }

void cpuoptical_(int *gpusize)
{
    if (!gpusize || !commons_present()) return report(FD2_ERR_STATE, nullptr, "cpuoptical_");
    const fd2_params p = params_from_common();
    fd2_ctx *c = nullptr;
    fd2_status s = fd2_create(&p, nullptr, &c);
    if (s == FD2_OK) s = submit_range(c, *gpusize, std::min(optical_.myctropt, FD2_GPUBUFSIZE));
    if (s == FD2_OK) s = fd2_run(c);
    if (s == FD2_OK) s = fd2_wait(c);
    if (s == FD2_OK) s = accumulate_into_commons(c);
    report(s, c, "cpuoptical_");
    fd2_destroy(c);
}

}  // extern "C"
