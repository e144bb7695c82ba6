// autotune.cu — shg_autotune: picks, per (precision, grid side) class, the compiled variant of
// the fused march (cluster split, threads per CTA) with the highest throughput on this
// device.  The reference fixes its launch shapes at compile time (src/cuSHG.cu:22-23) and
// has nothing to tune.
//
// The tuning batch: enough instances of the class to fill the device three times over for
// the variant with the most resident clusters, nz = 33 (32 steps), parameters spread like a
// sweep (waist, focus, power), so the timing sees the steady state of a persistent launch.
// Each variant runs once untimed, then three times between CUDA events; the median counts.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "shg_host.h"
#include "ssfm_variants.h"

using namespace shg;

extern "C" shg_status shg_autotune(int32_t precision, int32_t n, shg_tune_result* out) {
    clear_error();
    if (!out) return fail(SHG_ERR_INVALID, "out is NULL");
    if (precision != 32 && precision != 64) return fail(SHG_ERR_INVALID, "precision must be 32 or 64");
    const PlainVariant* cand[16];
    const int nc = plain_candidates(precision, n, cand, 16);
    if (nc == 0) return fail(SHG_ERR_UNSUPPORTED, "no kernel built for grid side %d at precision %d", n, precision);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(SHG_ERR_NO_DEVICE, "no CUDA device visible");
    }
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // instances: three device fills for the variant with the smallest cluster
    int cmin = 0;  // smallest cluster of the fused candidates (0: multi-pass only)
    for (int i = 0; i < nc; ++i)
        if (cand[i]->cluster > 0) cmin = cmin ? std::min(cmin, cand[i]->cluster) : cand[i]->cluster;
    const int count = cmin ? std::max(8, 3 * 2 * sms / cmin) : 8;
    shg_params base;
    shg_default_params(&base);
    base.nx = base.ny = n;
    base.nz = 33;
    base.precision = precision;
    base.lz = 10000.0;
    std::vector<InstDesc> descs(count);
    for (int i = 0; i < count; ++i) {
        shg_params q = base;
        const double u = (i + 0.5) / count;
        q.waist = 15.0 + 45.0 * u;
        q.lx = q.ly = 12.0 * q.waist;
        q.focus = q.lz * u;
        q.power = 1.0 + 49.0 * (1.0 - u);
        descs[i] = make_plain_desc(q, q.temp, q.temp);
        descs[i].slot = i;
    }
    cudaStream_t s = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
    void* buf = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    shg_status rc = SHG_OK;
    double rate[16] = {0};
    do {
        if ((e = dev_alloc((void**)&buf, sizeof(InstDesc) * (size_t)count + 256, s)) != cudaSuccess) {
            rc = cuda_fail(e, "cudaMallocAsync");
            break;
        }
        InstDesc* dd = reinterpret_cast<InstDesc*>(buf);
        int* queue = reinterpret_cast<int*>(dd + count);
        if ((e = cudaMemcpyAsync(dd, descs.data(), sizeof(InstDesc) * (size_t)count, cudaMemcpyHostToDevice, s)) !=
                cudaSuccess ||
            (e = cudaEventCreate(&ev[0])) != cudaSuccess || (e = cudaEventCreate(&ev[1])) != cudaSuccess) {
            rc = cuda_fail(e, "tuning set-up");
            break;
        }
        const double work = (double)count * n * n * (base.nz - 1);
        for (int c = 0; c < nc && rc == SHG_OK; ++c) {
            float ms[4] = {0, 0, 0, 0};
            for (int r = 0; r < 4; ++r) {
                if ((e = cudaMemsetAsync(queue, 0, sizeof(int), s)) != cudaSuccess ||
                    (e = cudaEventRecord(ev[0], s)) != cudaSuccess ||
                    (e = run_variant(cand[c], dd, descs.data(), count, queue, s)) != cudaSuccess ||
                    (e = cudaEventRecord(ev[1], s)) != cudaSuccess || (e = cudaEventSynchronize(ev[1])) != cudaSuccess ||
                    (e = cudaEventElapsedTime(&ms[r], ev[0], ev[1])) != cudaSuccess) {
                    rc = cuda_fail(e, "tuning launch");
                    break;
                }
            }
            std::sort(ms + 1, ms + 4);  // ms[0] is the untimed first run
            rate[c] = work / (ms[2] * 1e-3);
        }
    } while (0);
    for (cudaEvent_t x : ev)
        if (x) cudaEventDestroy(x);
    if (buf) cudaFreeAsync(buf, s);
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    if (rc != SHG_OK) return rc;
    int best = 0;
    for (int c = 1; c < nc; ++c)
        if (rate[c] > rate[best]) best = c;
    set_plain_choice(cand[best]);
    std::memset(out, 0, sizeof(*out));
    out->precision = precision;
    out->n = n;
    out->cluster = cand[best]->cluster;
    out->threads = cand[best]->threads;
    out->candidates = nc;
    out->pt_steps_per_s = rate[best];
    out->default_pt_steps_per_s = rate[0];
    return SHG_OK;
}

// shg_autotune_batch: the schedule of every grid-size class scored by the time of the whole
// given batch.  The classes of a mixed batch run side by side on forked streams and share
// the SMs, so the variant that is fastest for a class alone can slow the batch (a class that
// fills every SM with its own CTAs holds back the clusters of the larger classes).
// Coordinate descent from the compiled defaults: for each class, largest total work first,
// every other compiled variant is timed with the rest fixed and kept if the batch is at
// least 1 % faster.  A timing is the median of three runs of the batch (no field outputs,
// SH powers kept on the device) after one untimed run.
extern "C" shg_status shg_autotune_batch(const shg_params* params, int32_t count, shg_tune_result* out,
                                         int32_t max_out, int32_t* n_out) {
    clear_error();
    if (!params || count <= 0) return fail(SHG_ERR_INVALID, "params is NULL or count <= 0");
    if (!out || !n_out || max_out <= 0) return fail(SHG_ERR_INVALID, "out / n_out is NULL or max_out <= 0");
    for (int i = 0; i < count; ++i) {
        shg_status st = shg_check_params(&params[i]);
        if (st != SHG_OK) return fail(st, "instance %d: %s", i, shg_last_error());
        if (params[i].thermal) return fail(SHG_ERR_UNSUPPORTED, "instance %d: batched runs are plain (thermal == 0)", i);
        if (params[i].precision != params[0].precision)
            return fail(SHG_ERR_INVALID, "instance %d: all instances must share one precision", i);
        if (params[i].march != SHG_MARCH_AUTO)
            return fail(SHG_ERR_INVALID, "instance %d: the tuner chooses the march (march must be SHG_MARCH_AUTO)", i);
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(SHG_ERR_NO_DEVICE, "no CUDA device visible");
    }
    const int precision = params[0].precision;
    // the classes, by total work
    struct Cls { int n; double work; };
    std::vector<Cls> cls;
    double work = 0.0;
    for (int i = 0; i < count; ++i) {
        const double w = (double)params[i].nx * params[i].nx * shg_steps(&params[i]);
        work += w;
        auto it = std::find_if(cls.begin(), cls.end(), [&](const Cls& c) { return c.n == params[i].nx; });
        if (it == cls.end()) cls.push_back({params[i].nx, w});
        else it->work += w;
    }
    std::sort(cls.begin(), cls.end(), [](const Cls& a, const Cls& b) { return a.work > b.work; });
    if ((int)cls.size() > max_out) return fail(SHG_ERR_INVALID, "the batch has %d classes, out holds %d", (int)cls.size(), max_out);
    // start from the compiled defaults
    std::vector<std::vector<const PlainVariant*>> cand(cls.size());
    std::vector<int> pick(cls.size(), 0);
    for (size_t k = 0; k < cls.size(); ++k) {
        const PlainVariant* c[16];
        const int nc = plain_candidates(precision, cls[k].n, c, 16);
        cand[k].assign(c, c + nc);
        set_plain_choice(cand[k][0]);
    }
    cudaStream_t s = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
    cudaEvent_t ev[2] = {nullptr, nullptr};
    shg_status rc = SHG_OK;
    auto time_batch = [&](double* ms_out) -> shg_status {
        float ms[4] = {0, 0, 0, 0};
        for (int r = 0; r < 4; ++r) {
            if ((e = cudaEventRecord(ev[0], s)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
            shg_status st = plain_solve_batch(params, count, nullptr, nullptr, nullptr, s, nullptr, nullptr);
            if (st != SHG_OK) return st;
            if ((e = cudaEventRecord(ev[1], s)) != cudaSuccess || (e = cudaEventSynchronize(ev[1])) != cudaSuccess ||
                (e = cudaEventElapsedTime(&ms[r], ev[0], ev[1])) != cudaSuccess)
                return cuda_fail(e, "tuning run");
        }
        std::sort(ms + 1, ms + 4);  // ms[0] is the untimed first run
        *ms_out = ms[2];
        return SHG_OK;
    };
    double t_default = 0.0, t_best = 0.0;
    do {
        if ((e = cudaEventCreate(&ev[0])) != cudaSuccess || (e = cudaEventCreate(&ev[1])) != cudaSuccess) {
            rc = cuda_fail(e, "cudaEventCreate");
            break;
        }
        if ((rc = time_batch(&t_default)) != SHG_OK) break;
        t_best = t_default;
        for (size_t k = 0; k < cls.size() && rc == SHG_OK; ++k) {
            for (int c = 1; c < (int)cand[k].size() && rc == SHG_OK; ++c) {
                set_plain_choice(cand[k][c]);
                double t = 0.0;
                if ((rc = time_batch(&t)) != SHG_OK) break;
                if (t < 0.99 * t_best) {
                    t_best = t;
                    pick[k] = c;
                }
            }
            set_plain_choice(cand[k][pick[k]]);
        }
    } while (0);
    for (cudaEvent_t x : ev)
        if (x) cudaEventDestroy(x);
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    if (rc != SHG_OK) {
        for (size_t k = 0; k < cls.size(); ++k) set_plain_choice(cand[k][0]);
        return rc;
    }
    for (size_t k = 0; k < cls.size(); ++k) {
        shg_tune_result& r = out[k];
        std::memset(&r, 0, sizeof(r));
        r.precision = precision;
        r.n = cls[k].n;
        r.cluster = cand[k][pick[k]]->cluster;
        r.threads = cand[k][pick[k]]->threads;
        r.candidates = (int)cand[k].size();
        r.pt_steps_per_s = work / (t_best * 1e-3);
        r.default_pt_steps_per_s = work / (t_default * 1e-3);
    }
    *n_out = (int)cls.size();
    return SHG_OK;
}

extern "C" void shg_autotune_reset(void) { clear_plain_choices(); }

// shg_set_schedule: the compiled variant of a class chosen by its split, without timing (for
// example a schedule that shg_autotune_batch found in an earlier process).
extern "C" shg_status shg_set_schedule(int32_t precision, int32_t n, int32_t cluster, int32_t threads) {
    clear_error();
    if (precision != 32 && precision != 64) return fail(SHG_ERR_INVALID, "precision must be 32 or 64");
    const PlainVariant* cand[16];
    const int nc = plain_candidates(precision, n, cand, 16);
    for (int i = 0; i < nc; ++i)
        if (cand[i]->cluster == cluster && cand[i]->threads == threads) {
            set_plain_choice(cand[i]);
            return SHG_OK;
        }
    return fail(SHG_ERR_UNSUPPORTED, "no compiled variant of grid side %d at precision %d with %d-CTA clusters x %d threads",
                n, precision, cluster, threads);
}
