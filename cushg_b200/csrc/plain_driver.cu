// plain_driver.cu — host driver of plain (non-thermal) runs: one instance, or a batch of
// instances with uneven grid sizes and step counts.
//
// The batch replaces the one-process-per-point sweep of src/cuSHG.sh:58-94.  Instances are
// grouped by compiled variant (precision, grid side); each group is ONE persistent launch
// of the fused march, as many clusters as fit on the device, fed by a device work queue
// (an atomic counter over the group's descriptors, ordered longest march first, so the
// clusters drain it like a longest-processing-time schedule).  Groups run concurrently on
// forked streams, the largest total work first, so the smaller classes fill the SMs the
// largest one frees at its tail.  A batch plan (shg_batch_plan_*) captures the same
// sequence once into a CUDA graph and replays it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "shg_host.h"
#include "ssfm_variants.h"

namespace shg {

namespace {

// A few non-blocking streams per device, created once, for the forked group launches.
struct ForkStreams {
    static constexpr int kMax = 8;
    cudaStream_t s[kMax] = {};
    cudaEvent_t ev[kMax + 1] = {};
    bool ready = false;
};

std::mutex g_fork_mu;
ForkStreams g_fork[64];

cudaError_t fork_streams(int dev, ForkStreams** out) {
    std::lock_guard<std::mutex> lk(g_fork_mu);
    ForkStreams& f = g_fork[dev & 63];
    if (!f.ready) {
        for (int i = 0; i < ForkStreams::kMax; ++i) {
            cudaError_t e = cudaStreamCreateWithFlags(&f.s[i], cudaStreamNonBlocking);
            if (e != cudaSuccess) return e;
        }
        for (int i = 0; i <= ForkStreams::kMax; ++i) {
            cudaError_t e = cudaEventCreateWithFlags(&f.ev[i], cudaEventDisableTiming);
            if (e != cudaSuccess) return e;
        }
        f.ready = true;
    }
    *out = &f;
    return cudaSuccess;
}

}  // namespace

shg_status plain_solve_device(const shg_params& p, const void* signal_in, void* pump_out, void* signal_out,
                              shg_stats* stats, cudaStream_t stream, void* slices_p, void* slices_s,
                              const double* poling_dev) {
    int out32 = 0;
    const PlainVariant* v = plain_variant_of(p, &out32);
    if (!v) return fail(SHG_ERR_UNSUPPORTED, "no kernel for grid side %d", p.nx);
    InstDesc d = make_plain_desc(p, p.temp, p.temp);
    d.out32 = out32;
    d.signal_in = signal_in;
    d.has_signal_in = signal_in ? 1 : 0;
    d.pump_out = pump_out;
    d.signal_out = signal_out;
    d.slices_p = slices_p;
    d.slices_s = slices_s;
    d.nslices = (slices_p || slices_s) ? p.nz : 0;
    d.poling = poling_dev;
    cudaError_t e;
    void* buf = nullptr;
    const size_t bytes = sizeof(InstDesc) + 2 * sizeof(double);
    if ((e = dev_alloc((void**)&buf, bytes, stream)) != cudaSuccess) return cuda_fail(e, "cudaMallocAsync");
    InstDesc* dd = reinterpret_cast<InstDesc*>(buf);
    double* pw = reinterpret_cast<double*>(reinterpret_cast<char*>(buf) + sizeof(InstDesc));
    d.power_out = pw;
    shg_status rc = SHG_OK;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    do {
        if ((e = cudaMemcpyAsync(dd, &d, sizeof(d), cudaMemcpyHostToDevice, stream)) != cudaSuccess) {
            rc = cuda_fail(e, "cudaMemcpyAsync desc");
            break;
        }
        if (stats) {
            cudaEventCreate(&t0);
            cudaEventCreate(&t1);
            cudaEventRecord(t0, stream);
        }
        if ((e = run_variant(v, dd, &d, 1, nullptr, stream)) != cudaSuccess) { rc = cuda_fail(e, "launch ssfm_plain_kernel"); break; }
        if (stats) {
            cudaEventRecord(t1, stream);
            double h[2] = {0, 0};
            if ((e = cudaMemcpyAsync(h, pw, sizeof(h), cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
                (e = cudaStreamSynchronize(stream)) != cudaSuccess) {
                rc = cuda_fail(e, "ssfm_plain_kernel");
                break;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, t0, t1);
            std::memset(stats, 0, sizeof(*stats));
            stats->sh_power = h[0];
            stats->pump_power = h[1];
            stats->steps = d.nsteps;
            stats->outer_iterations = 1;
            stats->device_ms = ms;
            if (!std::isfinite(h[0]) || !std::isfinite(h[1]))
                rc = fail(SHG_ERR_NONFINITE, "SH / pump power %g / %g", h[0], h[1]);
        }
    } while (0);
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    cudaFreeAsync(buf, stream);
    e = cudaGetLastError();
    if (rc == SHG_OK && e != cudaSuccess) rc = cuda_fail(e, "plain run");
    return rc;
}

// Batch layout: instances grouped by variant (longest march first inside a group), groups
// ordered by total work, descriptors in that order.
struct BatchLayout {
    struct Group {
        const PlainVariant* v;
        int begin, end;
        double work;
    };
    std::vector<InstDesc> descs;  // execution order
    std::vector<Group> groups;
};

static BatchLayout batch_layout(const shg_params* params, int count, void* const* pump_out, void* const* signal_out,
                                double* power_slots) {
    struct Item { const PlainVariant* v; int idx; double cost; int out32; };
    std::vector<Item> items(count);
    for (int i = 0; i < count; ++i) {
        int out32 = 0;
        const PlainVariant* v = plain_variant_of(params[i], &out32);
        items[i] = {v, i, (double)params[i].nx * params[i].nx * shg_steps(&params[i]), out32};
    }
    std::stable_sort(items.begin(), items.end(), [](const Item& a, const Item& b) {
        if (a.v != b.v) return a.v < b.v;
        return a.cost > b.cost;
    });
    BatchLayout L;
    L.descs.resize(count);
    for (int k = 0; k < count; ++k) {
        const int i = items[k].idx;
        InstDesc d = make_plain_desc(params[i], params[i].temp, params[i].temp);
        d.slot = i;
        d.out32 = items[k].out32;
        d.pump_out = pump_out ? pump_out[i] : nullptr;
        d.signal_out = signal_out ? signal_out[i] : nullptr;
        d.power_out = power_slots + 2 * (size_t)i;
        L.descs[k] = d;
    }
    for (int k = 0; k < count;) {
        int j = k;
        double w = 0;
        while (j < count && items[j].v == items[k].v) w += items[j++].cost;
        L.groups.push_back({items[k].v, k, j, w});
        k = j;
    }
    // The groups an FP32 batch's guard promotes to the FP64 march go first: few instances, but
    // each runs about 2.5x as long as in FP32, so they are the batch's longest jobs; launched
    // last, their clusters would wait for SMs and trail the FP32 groups.  Then by total work.
    std::sort(L.groups.begin(), L.groups.end(), [&](const BatchLayout::Group& a, const BatchLayout::Group& b) {
        const bool pa = a.v->precision > params[0].precision, pb = b.v->precision > params[0].precision;
        if (pa != pb) return pa;
        return a.work > b.work;
    });
    return L;
}

// Device-to-host copies of a group's output fields (host arrays indexed by batch slot),
// enqueued on the stream that ran the group so that they overlap the other groups' marches.
struct HostOutputs {
    void* const* pump;
    void* const* signal;
};

static cudaError_t copy_group_outputs(const BatchLayout& L, const BatchLayout::Group& G, const HostOutputs* ho,
                                      size_t cbytes, cudaStream_t s) {
    if (!ho) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    for (int k = G.begin; k < G.end && e == cudaSuccess; ++k) {
        const InstDesc& d = L.descs[k];
        const size_t bytes = (size_t)d.n * d.n * cbytes;
        if (ho->pump && ho->pump[d.slot] && d.pump_out)
            e = cudaMemcpyAsync(ho->pump[d.slot], d.pump_out, bytes, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && ho->signal && ho->signal[d.slot] && d.signal_out)
            e = cudaMemcpyAsync(ho->signal[d.slot], d.signal_out, bytes, cudaMemcpyDeviceToHost, s);
    }
    return e;
}

// Enqueue the batched march on `stream`: zero the groups' work-queue counters, then one
// persistent launch per group, the groups on the fork streams `fs` (joined back into
// `stream`) when there are several, each followed on its stream by the copies of its outputs
// to the host when `ho` is given.  Capturable into a CUDA graph (without host copies).
static cudaError_t enqueue_batch(const BatchLayout& L, const InstDesc* dd, int* queues, cudaStream_t stream,
                                 cudaStream_t* fs, cudaEvent_t* ev, int nfork, const HostOutputs* ho = nullptr,
                                 size_t cbytes = 0) {
    cudaError_t e;
    const int ng = (int)L.groups.size();
    if ((e = cudaMemsetAsync(queues, 0, sizeof(int) * (size_t)ng, stream)) != cudaSuccess) return e;
    if (ng == 1) {
        if ((e = run_variant(L.groups[0].v, dd + L.groups[0].begin, L.descs.data() + L.groups[0].begin,
                             L.groups[0].end - L.groups[0].begin, queues, stream)) != cudaSuccess)
            return e;
        return copy_group_outputs(L, L.groups[0], ho, cbytes, stream);
    }
    const int nf = std::min(ng, nfork);
    if ((e = cudaEventRecord(ev[nfork], stream)) != cudaSuccess) return e;
    for (int g = 0; g < nf; ++g)
        if ((e = cudaStreamWaitEvent(fs[g], ev[nfork], 0)) != cudaSuccess) return e;
    for (int g = 0; g < ng; ++g) {
        const BatchLayout::Group& G = L.groups[g];
        if ((e = run_variant(G.v, dd + G.begin, L.descs.data() + G.begin, G.end - G.begin, queues + g, fs[g % nf])) !=
                cudaSuccess ||
            (e = copy_group_outputs(L, G, ho, cbytes, fs[g % nf])) != cudaSuccess)
            return e;
    }
    for (int g = 0; g < nf; ++g) {
        if ((e = cudaEventRecord(ev[g], fs[g])) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(stream, ev[g], 0)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Host-to-device upload of a batch's descriptors through page-locked staging.  A copy from
// pageable memory may make the driver wait for the stream to drain before it stages the data,
// which would hold the host until the previous batch on the stream has finished and leave the
// GPU idle while the host prepares the next one.  A small ring of page-locked slots, each
// reused only after the copy that last read it has completed, keeps the call asynchronous.
// While the stream is being captured the plain copy is used.
class PinnedStage {
  public:
    cudaError_t upload(void* dst, const void* src, size_t bytes, cudaStream_t s) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
            cudaGetLastError();
            return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
        }
        std::lock_guard<std::mutex> lk(mu_);
        Slot& sl = slots_[next_];
        next_ = (next_ + 1) % kSlots;
        cudaError_t e;
        if (sl.done) {
            if ((e = cudaEventSynchronize(sl.done)) != cudaSuccess) return e;
            cudaEventDestroy(sl.done);  // recreated below on the current device
            sl.done = nullptr;
        }
        if (sl.cap < bytes) {
            if (sl.buf) cudaFreeHost(sl.buf);
            sl.buf = nullptr;
            sl.cap = 0;
            if ((e = cudaHostAlloc(&sl.buf, bytes, cudaHostAllocPortable)) != cudaSuccess) return e;
            sl.cap = bytes;
        }
        std::memcpy(sl.buf, src, bytes);
        if ((e = cudaMemcpyAsync(dst, sl.buf, bytes, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
        if ((e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming)) != cudaSuccess) return e;
        return cudaEventRecord(sl.done, s);
    }

  private:
    static constexpr int kSlots = 4;
    struct Slot {
        void* buf = nullptr;
        size_t cap = 0;
        cudaEvent_t done = nullptr;
    };
    Slot slots_[kSlots];
    int next_ = 0;
    std::mutex mu_;
};

static PinnedStage g_desc_stage;  // process lifetime; its page-locked slots are held until exit

static size_t batch_bytes(int count) {
    return sizeof(InstDesc) * (size_t)count + 2 * sizeof(double) * (size_t)count + sizeof(int) * 64;
}

shg_status plain_solve_batch(const shg_params* params, int count, void* const* pump_out, void* const* signal_out,
                             double* sh_power_out, cudaStream_t stream, void* const* pump_host,
                             void* const* signal_host) {
    if (count == 0) return SHG_OK;
    cudaError_t e;
    void* buf = nullptr;
    if ((e = dev_alloc((void**)&buf, batch_bytes(count), stream)) != cudaSuccess) return cuda_fail(e, "cudaMallocAsync");
    InstDesc* dd = reinterpret_cast<InstDesc*>(buf);
    double* pw = reinterpret_cast<double*>(dd + count);
    int* queues = reinterpret_cast<int*>(pw + 2 * (size_t)count);
    const BatchLayout L = batch_layout(params, count, pump_out, signal_out, pw);
    shg_status rc = SHG_OK;
    do {
        if (L.groups.size() > 64) { rc = fail(SHG_ERR_UNSUPPORTED, "more than 64 kernel variants in one batch"); break; }
        if ((e = g_desc_stage.upload(dd, L.descs.data(), sizeof(InstDesc) * (size_t)count, stream)) != cudaSuccess) {
            rc = cuda_fail(e, "descriptor upload");
            break;
        }
        int dev = 0;
        cudaGetDevice(&dev);
        ForkStreams* f = nullptr;
        if ((e = fork_streams(dev, &f)) != cudaSuccess) { rc = cuda_fail(e, "stream pool"); break; }
        const HostOutputs ho = {pump_host, signal_host};
        const bool copies = pump_host || signal_host;
        if ((e = enqueue_batch(L, dd, queues, stream, f->s, f->ev, ForkStreams::kMax, copies ? &ho : nullptr,
                               complex_bytes(params[0]))) != cudaSuccess) {
            rc = cuda_fail(e, "launch ssfm_plain_kernel");
            break;
        }
        if (sh_power_out) {
            std::vector<double> h(2 * (size_t)count);
            if ((e = cudaMemcpyAsync(h.data(), pw, sizeof(double) * 2 * (size_t)count, cudaMemcpyDeviceToHost, stream)) !=
                    cudaSuccess ||
                (e = cudaStreamSynchronize(stream)) != cudaSuccess) {
                rc = cuda_fail(e, "batch run");
                break;
            }
            for (int i = 0; i < count; ++i) sh_power_out[i] = h[2 * (size_t)i];
            for (int i = 0; i < count && rc == SHG_OK; ++i)
                if (!std::isfinite(h[2 * (size_t)i]) || !std::isfinite(h[2 * (size_t)i + 1]))
                    rc = fail(SHG_ERR_NONFINITE, "instance %d: SH / pump power %g / %g", i, h[2 * (size_t)i],
                              h[2 * (size_t)i + 1]);
        }
    } while (0);
    cudaFreeAsync(buf, stream);
    e = cudaGetLastError();
    if (rc == SHG_OK && e != cudaSuccess) rc = cuda_fail(e, "batch run");
    return rc;
}

}  // namespace shg

// ------------------------------------------------------------------ batch plans (graphs)
struct shg_batch_plan {
    int count = 0;
    int device = 0;
    void* buf = nullptr;          // descriptors, power slots, queue counters (cudaMalloc)
    double* powers = nullptr;     // device, [2 * count]
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t fork[shg::ForkStreams::kMax] = {};
    cudaEvent_t ev[shg::ForkStreams::kMax + 1] = {};
};

using namespace shg;

static void plan_release(shg_batch_plan* P) {
    if (!P) return;
    if (P->exec) cudaGraphExecDestroy(P->exec);
    if (P->graph) cudaGraphDestroy(P->graph);
    for (cudaStream_t s : P->fork)
        if (s) cudaStreamDestroy(s);
    for (cudaEvent_t e : P->ev)
        if (e) cudaEventDestroy(e);
    if (P->buf) cudaFree(P->buf);
    delete P;
}

extern "C" shg_status shg_batch_plan_create(const shg_params* params, int32_t count, void* const* pump_out_dev,
                                            void* const* signal_out_dev, shg_batch_plan** plan) {
    clear_error();
    if (!plan) return fail(SHG_ERR_INVALID, "plan is NULL");
    *plan = nullptr;
    if (!params || count <= 0) return fail(SHG_ERR_INVALID, "params is NULL or count <= 0");
    for (int i = 0; i < count; ++i) {
        shg_status st = shg_check_params(&params[i]);
        if (st != SHG_OK) return fail(st, "instance %d: %s", i, shg_last_error());
        if (params[i].thermal) return fail(SHG_ERR_UNSUPPORTED, "instance %d: batched runs are plain (thermal == 0)", i);
        if (params[i].precision != params[0].precision)
            return fail(SHG_ERR_INVALID, "instance %d: all instances must share one precision", i);
    }
    shg_batch_plan* P = new shg_batch_plan;
    P->count = count;
    cudaError_t e;
    shg_status rc = SHG_OK;
    cudaStream_t cap = nullptr;
    do {
        if ((e = cudaGetDevice(&P->device)) != cudaSuccess) { rc = cuda_fail(e, "cudaGetDevice"); break; }
        if ((e = cudaMalloc(&P->buf, batch_bytes(count))) != cudaSuccess) { rc = cuda_fail(e, "cudaMalloc"); break; }
        InstDesc* dd = reinterpret_cast<InstDesc*>(P->buf);
        P->powers = reinterpret_cast<double*>(dd + count);
        int* queues = reinterpret_cast<int*>(P->powers + 2 * (size_t)count);
        const BatchLayout L = batch_layout(params, count, pump_out_dev, signal_out_dev, P->powers);
        if (L.groups.size() > 64) { rc = fail(SHG_ERR_UNSUPPORTED, "more than 64 kernel variants in one batch"); break; }
        if ((e = cudaMemcpy(dd, L.descs.data(), sizeof(InstDesc) * (size_t)count, cudaMemcpyHostToDevice)) != cudaSuccess) {
            rc = cuda_fail(e, "cudaMemcpy descriptors");
            break;
        }
        for (auto& s : P->fork)
            if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess) break;
        if (e == cudaSuccess)
            for (auto& ev : P->ev)
                if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) break;
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
        if (e != cudaSuccess) { rc = cuda_fail(e, "plan streams"); break; }
        // a first launch outside the capture sets the kernels' attributes and sizes
        for (const auto& G : L.groups)
            if ((e = run_variant(G.v, dd + G.begin, L.descs.data() + G.begin, 0, queues, cap)) != cudaSuccess) break;
        if (e != cudaSuccess) { rc = cuda_fail(e, "kernel set-up"); break; }
        if ((e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) {
            rc = cuda_fail(e, "cudaStreamBeginCapture");
            break;
        }
        const cudaError_t ee = enqueue_batch(L, dd, queues, cap, P->fork, P->ev, ForkStreams::kMax);
        e = cudaStreamEndCapture(cap, &P->graph);
        if (ee != cudaSuccess) { rc = cuda_fail(ee, "capture of the batched march"); break; }
        if (e != cudaSuccess) { rc = cuda_fail(e, "cudaStreamEndCapture"); break; }
        if ((e = cudaGraphInstantiate(&P->exec, P->graph, 0)) != cudaSuccess) {
            rc = cuda_fail(e, "cudaGraphInstantiate");
            break;
        }
    } while (0);
    if (cap) cudaStreamDestroy(cap);
    if (rc != SHG_OK) {
        plan_release(P);
        return rc;
    }
    *plan = P;
    return SHG_OK;
}

extern "C" shg_status shg_batch_plan_launch(shg_batch_plan* plan, void* stream) {
    clear_error();
    if (!plan || !plan->exec) return fail(SHG_ERR_INVALID, "plan is NULL");
    const cudaError_t e = cudaGraphLaunch(plan->exec, (cudaStream_t)stream);
    return e == cudaSuccess ? SHG_OK : cuda_fail(e, "cudaGraphLaunch");
}

extern "C" shg_status shg_batch_plan_powers(shg_batch_plan* plan, double* sh_power_out, void* stream) {
    clear_error();
    if (!plan || !sh_power_out) return fail(SHG_ERR_INVALID, "plan or sh_power_out is NULL");
    std::vector<double> h(2 * (size_t)plan->count);
    cudaError_t e;
    if ((e = cudaMemcpyAsync(h.data(), plan->powers, sizeof(double) * h.size(), cudaMemcpyDeviceToHost,
                             (cudaStream_t)stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize((cudaStream_t)stream)) != cudaSuccess)
        return cuda_fail(e, "plan powers");
    for (int i = 0; i < plan->count; ++i) sh_power_out[i] = h[2 * (size_t)i];
    return SHG_OK;
}

extern "C" void shg_batch_plan_destroy(shg_batch_plan* plan) {
    if (!plan) return;
    cudaDeviceSynchronize();
    plan_release(plan);
}
