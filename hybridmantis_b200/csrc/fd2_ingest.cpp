// fd2_ingest.cpp -- streaming event ingest (fd2_ingest_* in include/fd2.h).
//
// The reference's EDE tally fills a COMMON buffer of events and, each time
// it is full, calls gpuoptical_, which converts, copies, transports and
// tallies that buffer before PENELOPE may go on
// (main/hybridMANTIS_tallyEnergyDepositionEvents.f:171-310,
// main/hybridMANTIS_cuda_ver1_0.cu:107-446).  Here the producer goes on at
// once.  Two pinned staging batches alternate: while the GPU transports
// batch k, the host fills batch k+1; a full batch is copied on its own
// stream and the context's stream takes it over when the copy is done:
//
//   copy stream:  [H2D k]        [H2D k+1]             waits prep k-1
//   ctx stream:        [prep k | count, scan, fill | transport k] [prep k+1 ...
//
// A staging batch is refilled once its previous copy has finished (host
// waits on h2d[b]); a device staging batch is overwritten once the prep
// kernel that read it has run (copy stream waits on prep[b]).  The event
// arrays of the context are rewritten by prep k+1 after transport k on the
// same stream.  Event indices continue across batches (options.event_base +
// events so far) and the run counter stays fixed until fd2_ingest_end, so
// every photon draws what it would in one submission of the whole stream.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "fd2.h"
#include "fd2_ctx.h"
#include "fd2_host.h"
#include "fd2_internal.h"

using fd2::api::fail;

struct fd2_ingest {
    fd2_ctx *c = nullptr;
    int units = FD2_UNITS_CM;
    int64_t cap = 0;    // events per staging batch
    size_t esz = 0;     // bytes of one coordinate or energy (8 for cm, 4 for um)
    char *h[2] = {nullptr, nullptr};
    char *d[2] = {nullptr, nullptr};
    cudaEvent_t h2d[2] = {nullptr, nullptr}, prep[2] = {nullptr, nullptr};
    bool h2d_pending[2] = {false, false}, prep_pending[2] = {false, false};
    cudaStream_t copy = nullptr;
    int cur = 0;
    int64_t fill = 0;
    double mu = 0.0;  // photon mean of the batch being filled
    int64_t events = 0, batches = 0, base0 = 0;
    unsigned long long gen0 = 0;
    bool window_set = false;
    fd2_status err = FD2_OK;
    double wait_s = 0.0;
    std::chrono::steady_clock::time_point t0;
};

namespace {

fd2_status ingest_cuda(fd2_ingest *in, cudaError_t e, const char *what)
{
    const fd2_status s = e == cudaErrorMemoryAllocation ? FD2_ERR_OUT_OF_MEMORY : FD2_ERR_CUDA;
    in->err = fail(in->c, s, std::string("ingest: ") + what + ": " + cudaGetErrorString(e));
    return in->err;
}

#define IN_CUDA(in, call)                                          \
    do {                                                           \
        const cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return ingest_cuda(in, e_, #call);  \
    } while (0)

// Field f (0..3: x, y, z, energy; 4: history) of staging batch `base`.
inline char *field(const fd2_ingest *in, char *base, int f) { return base + (size_t)f * (size_t)in->cap * in->esz; }

// Make the current host batch writable: its previous copy must be done.
fd2_status acquire(fd2_ingest *in)
{
    const int b = in->cur;
    if (in->h2d_pending[b]) {
        const auto t0 = std::chrono::steady_clock::now();
        IN_CUDA(in, cudaEventSynchronize(in->h2d[b]));
        in->wait_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        in->h2d_pending[b] = false;
    }
    return FD2_OK;
}

// Copy the current batch to the GPU and queue its transport.
fd2_status launch(fd2_ingest *in)
{
    fd2_ctx *c = in->c;
    const int64_t n = in->fill;
    if (n == 0) return FD2_OK;
    const int b = in->cur;
    const size_t nb = (size_t)n;
    if (!in->window_set) {
        // shared-memory PRF window around the first batch's events (a tally
        // cache only: the results do not depend on it)
        std::vector<float> xs(nb), ys(nb);
        for (size_t i = 0; i < nb; ++i) {
            if (in->units == FD2_UNITS_CM) {
                xs[i] = (float)(((const double *)field(in, in->h[b], 0))[i] * (double)10000.0f);
                ys[i] = (float)(((const double *)field(in, in->h[b], 1))[i] * (double)10000.0f);
            } else {
                xs[i] = ((const float *)field(in, in->h[b], 0))[i];
                ys[i] = ((const float *)field(in, in->h[b], 1))[i];
            }
        }
        fd2::api::choose_window(c, xs.data(), ys.data(), nullptr, n);
        IN_CUDA(in, fd2::prepare_transport(c->cfg, 1));
        in->window_set = true;
    }
    // work-queue capacity for this batch; growing it frees the old queue, so
    // the transports still reading it finish first
    c->n_events = n;
    c->mu_total = in->mu;
    const double bound = in->mu * 1.01 + 10.0 * std::sqrt(in->mu) + 4096.0;
    const int64_t need = n + (int64_t)std::ceil(bound / (double)c->cfg.chunk) + 1024;
    if (need > c->chunk_cap) {
        IN_CUDA(in, cudaStreamSynchronize(c->stream));
        c->mu_total = in->mu * 1.5;  // headroom for later batches
        fd2_status st = fd2::api::ensure_chunks(c);
        c->mu_total = in->mu;
        if (st != FD2_OK) return in->err = st;
    }
    // H2D on the copy stream, once the prep kernel that last read d[b] ran
    if (in->prep_pending[b]) IN_CUDA(in, cudaStreamWaitEvent(in->copy, in->prep[b], 0));
    for (int f = 0; f < 5; ++f) {
        const size_t bytes = nb * (f < 4 ? in->esz : sizeof(int32_t));
        IN_CUDA(in, cudaMemcpyAsync(field(in, in->d[b], f), field(in, in->h[b], f), bytes, cudaMemcpyHostToDevice,
                                    in->copy));
    }
    IN_CUDA(in, cudaEventRecord(in->h2d[b], in->copy));
    in->h2d_pending[b] = true;
    // the context's stream: convert into the event arrays, then the run
    IN_CUDA(in, cudaStreamWaitEvent(c->stream, in->h2d[b], 0));
    if (in->units == FD2_UNITS_CM) {
        IN_CUDA(in, fd2::launch_prep_cm(c->stream, n, (const double *)field(in, in->d[b], 0),
                                        (const double *)field(in, in->d[b], 1), (const double *)field(in, in->d[b], 2),
                                        (const double *)field(in, in->d[b], 3), (const int32_t *)field(in, in->d[b], 4),
                                        c->n_prim, c->d_ev_pos, c->d_ev_e, c->d_ev_xyz, c->d_flags));
    } else {
        IN_CUDA(in, fd2::launch_prep_um(c->stream, n, (const float *)field(in, in->d[b], 0),
                                        (const float *)field(in, in->d[b], 1), (const float *)field(in, in->d[b], 2),
                                        (const float *)field(in, in->d[b], 3), (const int32_t *)field(in, in->d[b], 4),
                                        c->n_prim, c->d_ev_pos, c->d_ev_e, c->d_ev_xyz, c->d_flags));
    }
    IN_CUDA(in, cudaEventRecord(in->prep[b], c->stream));
    in->prep_pending[b] = true;
    c->opt.event_base = in->base0 + in->events;
    IN_CUDA(in, fd2::api::enqueue_segment(c, 0));
    IN_CUDA(in, fd2::api::enqueue_segment(c, 1));
    in->events += n;
    in->batches += 1;
    in->fill = 0;
    in->mu = 0.0;
    in->cur ^= 1;
    return FD2_OK;
}

template <typename T>
fd2_status push(fd2_ingest *in, const T *x, const T *y, const T *z, const T *e, const int32_t *hist, int64_t n)
{
    if (!in) return FD2_ERR_INVALID_ARGUMENT;
    if (in->err != FD2_OK) return in->err;
    if (n < 0 || (n > 0 && (!x || !y || !z || !e || !hist)))
        return fail(in->c, FD2_ERR_INVALID_ARGUMENT, "ingest push: null array or negative count");
    if (sizeof(T) != in->esz) return fail(in->c, FD2_ERR_INVALID_ARGUMENT, "ingest push: units differ from the ingest's");
    const double yield = in->c->params.yield;
    int64_t i = 0;
    while (i < n) {
        if (in->fill == 0) {
            fd2_status st = acquire(in);
            if (st != FD2_OK) return st;
        }
        const int64_t k = std::min(n - i, in->cap - in->fill);
        const size_t at = (size_t)in->fill, kb = (size_t)k;
        char *hb = in->h[in->cur];
        std::memcpy((T *)field(in, hb, 0) + at, x + i, kb * sizeof(T));
        std::memcpy((T *)field(in, hb, 1) + at, y + i, kb * sizeof(T));
        std::memcpy((T *)field(in, hb, 2) + at, z + i, kb * sizeof(T));
        std::memcpy((T *)field(in, hb, 3) + at, e + i, kb * sizeof(T));
        std::memcpy((int32_t *)field(in, hb, 4) + at, hist + i, kb * sizeof(int32_t));
        // the photon mean bounds the work-queue size (as fd2_submit_events)
        for (int64_t j = i; j < i + k; ++j)
            if (e[j] > 0) in->mu += (double)e[j] * yield;
        in->fill += k;
        i += k;
        if (in->fill == in->cap) {
            fd2_status st = launch(in);
            if (st != FD2_OK) return st;
        }
    }
    return FD2_OK;
}

void release(fd2_ingest *in)
{
    fd2_ctx *c = in->c;
    cudaSetDevice(c->device);
    if (in->copy) cudaStreamSynchronize(in->copy);
    cudaStreamSynchronize(c->stream);
    for (int b = 0; b < 2; ++b) {
        if (in->h[b]) cudaFreeHost(in->h[b]);
        if (in->d[b]) cudaFree(in->d[b]);
        if (in->h2d[b]) cudaEventDestroy(in->h2d[b]);
        if (in->prep[b]) cudaEventDestroy(in->prep[b]);
    }
    if (in->copy) cudaStreamDestroy(in->copy);
    c->opt.event_base = in->base0;
    c->n_events = 0;
    c->mu_total = 0.0;
    c->counts_ready = false;
    c->graph_valid = false;
    c->ingest_active = false;
    c->ingest = nullptr;
    delete in;
}

}  // namespace

extern "C" {

fd2_status fd2_ingest_begin(fd2_ctx *c, int64_t batch_events, int32_t units, fd2_ingest **out)
{
    if (!c || !out) return FD2_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (c->ingest_active) return fail(c, FD2_ERR_STATE, "an event ingest is already open");
    if (batch_events <= 0 || batch_events >= ((int64_t)1 << 31))
        return fail(c, FD2_ERR_INVALID_ARGUMENT, "ingest: batch_events out of range");
    if (units != FD2_UNITS_CM && units != FD2_UNITS_UM) return fail(c, FD2_ERR_INVALID_ARGUMENT, "ingest: units");
    if (c->geoms.size() != 1) return fail(c, FD2_ERR_STATE, "ingest is for a single geometry");
    if (c->opt.count_mode == FD2_COUNT_GIVEN) return fail(c, FD2_ERR_STATE, "ingest samples photon counts; count_mode GIVEN");
    if (c->run_pending) {
        const fd2_status w = fd2_wait(c);
        if (w != FD2_OK) return w;
    }
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(c, FD2_ERR_CUDA, "ingest: cudaSetDevice");
    fd2_status st = fd2::api::check_status(c);  // clears a stale status word
    if (st != FD2_OK) return st;
    if ((st = fd2::api::ensure_events(c, batch_events)) != FD2_OK) return st;
    fd2_ingest *in = new fd2_ingest;
    in->c = c;
    in->units = units;
    in->cap = batch_events;
    in->esz = units == FD2_UNITS_CM ? sizeof(double) : sizeof(float);
    in->base0 = c->opt.event_base;
    in->t0 = std::chrono::steady_clock::now();
    c->ingest_active = true;
    c->ingest = in;
    auto bail = [&](cudaError_t e, const char *what) {
        ingest_cuda(in, e, what);
        const fd2_status s = in->err;
        release(in);
        return s;
    };
    const size_t bytes = (size_t)batch_events * (4 * in->esz + sizeof(int32_t));
    cudaError_t e = cudaSuccess;
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
        e = cudaHostAlloc((void **)&in->h[b], bytes, cudaHostAllocDefault);
        if (e == cudaSuccess) e = cudaMalloc((void **)&in->d[b], bytes);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&in->h2d[b], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&in->prep[b], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&in->copy, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(e, "staging buffers");
    // photons counted before the stream (the stream's total is the difference)
    e = cudaMemcpy(&in->gen0, c->d_gen_total, sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    // the stream is one submission: its run counter starts at 0 (as fd2_submit_events)
    if (e == cudaSuccess) e = cudaMemsetAsync(c->d_flags + 1, 0, sizeof(int), c->stream);
    if (e == cudaSuccess) e = cudaEventRecord(c->ev_start, c->stream);
    if (e == cudaSuccess) e = cudaEventRecord(c->ev_t0, c->stream);
    if (e != cudaSuccess) return bail(e, "ingest start");
    c->graph_valid = false;
    *out = in;
    return FD2_OK;
}

fd2_status fd2_ingest_push(fd2_ingest *in, const double *x_cm, const double *y_cm, const double *z_cm,
                           const double *de_ev, const int32_t *hist, int64_t n)
{
    return push<double>(in, x_cm, y_cm, z_cm, de_ev, hist, n);
}

fd2_status fd2_ingest_push_um(fd2_ingest *in, const float *x_um, const float *y_um, const float *z_um,
                              const float *e_ev, const int32_t *hist, int64_t n)
{
    return push<float>(in, x_um, y_um, z_um, e_ev, hist, n);
}

fd2_status fd2_ingest_file(fd2_ingest *in, const char *path)
{
    if (!in || !path) return FD2_ERR_INVALID_ARGUMENT;
    if (in->err != FD2_OK) return in->err;
    if (in->units == FD2_UNITS_CM) {
        return fd2host::stream_events_text(
            path, in->cap, [&](const double *x, const double *y, const double *z, const double *e, const int32_t *h,
                               int64_t n) { return fd2_ingest_push(in, x, y, z, e, h, n); });
    }
    return fd2host::stream_events_binary(
        path, in->cap, nullptr,
        [&](const float *x, const float *y, const float *z, const float *e, const int32_t *h, const uint16_t *g,
            int64_t n) {
            if (g)
                for (int64_t i = 0; i < n; ++i)
                    if (g[i] != 0) return fail(in->c, FD2_ERR_INVALID_ARGUMENT, "ingest: geometry ids other than 0");
            return fd2_ingest_push_um(in, x, y, z, e, h, n);
        });
}

fd2_status fd2_ingest_end(fd2_ingest *in, fd2_ingest_stats *stats)
{
    if (!in) return FD2_ERR_INVALID_ARGUMENT;
    fd2_ctx *c = in->c;
    cudaSetDevice(c->device);
    fd2_status st = in->err;
    if (st == FD2_OK) st = launch(in);
    if (st == FD2_OK) {
        // PHS from the whole stream's per-history counts, then the next run
        // counter; fd2_wait keeps the deadline and the abort path of a run
        cudaError_t e = fd2::api::enqueue_segment(c, 2);
        if (e == cudaSuccess) e = cudaEventRecord(c->ev_t1, c->stream);
        if (e == cudaSuccess) e = cudaEventRecord(c->ev_end, c->stream);
        if (e != cudaSuccess) {
            st = ingest_cuda(in, e, "ingest end");
        } else {
            c->run_pending = true;
            c->ran_once = true;
            st = fd2_wait(c);
        }
    }
    unsigned long long gen1 = in->gen0;
    if (st == FD2_OK) {
        const cudaError_t e = cudaMemcpy(&gen1, c->d_gen_total, sizeof gen1, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) st = ingest_cuda(in, e, "photon total");
    }
    c->last_photons = (int64_t)(gen1 - in->gen0);
    if (stats) {
        std::memset(stats, 0, sizeof *stats);
        stats->events = in->events;
        stats->batches = in->batches;
        stats->photons = (int64_t)(gen1 - in->gen0);
        stats->push_wait_seconds = in->wait_s;
        if (st == FD2_OK) cudaEventElapsedTime(&stats->device_ms, c->ev_start, c->ev_end);
    }
    const auto t0 = in->t0;
    release(in);
    if (stats) stats->host_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return st;
}

}  // extern "C"
