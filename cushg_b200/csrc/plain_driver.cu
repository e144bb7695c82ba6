// plain_driver.cu — host driver of plain (non-thermal) runs: one instance, or a batch of
// instances with uneven grid sizes and step counts.
//
// The batch replaces the one-process-per-point sweep of src/cuSHG.sh:58-94: instances are
// grouped by compiled variant (precision, grid side), each group is one launch of the
// fused march with one cluster per instance, groups run concurrently on forked streams,
// and inside a group instances are ordered longest-first so the block scheduler packs
// the SMs like a longest-processing-time queue.
#include <cuda_runtime.h>

#include <algorithm>
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
    const PlainVariant* v = find_plain_variant(p.precision, p.nx);
    if (!v) return fail(SHG_ERR_UNSUPPORTED, "no kernel for grid side %d", p.nx);
    InstDesc d = make_plain_desc(p, p.temp, p.temp);
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
    if ((e = cudaMallocAsync(&buf, bytes, stream)) != cudaSuccess) return cuda_fail(e, "cudaMallocAsync");
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
        if ((e = v->launch(dd, 1, stream)) != cudaSuccess) { rc = cuda_fail(e, "launch ssfm_plain_kernel"); break; }
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
        }
    } while (0);
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    cudaFreeAsync(buf, stream);
    e = cudaGetLastError();
    if (rc == SHG_OK && e != cudaSuccess) rc = cuda_fail(e, "plain run");
    return rc;
}

shg_status plain_solve_batch(const shg_params* params, int count, void* const* pump_out, void* const* signal_out,
                             double* sh_power_out, cudaStream_t stream) {
    if (count == 0) return SHG_OK;
    // group by variant, longest march first inside a group
    struct Item { const PlainVariant* v; int idx; double cost; };
    std::vector<Item> items(count);
    for (int i = 0; i < count; ++i) {
        const PlainVariant* v = find_plain_variant(params[i].precision, params[i].nx);
        items[i] = {v, i, (double)params[i].nx * params[i].nx * shg_steps(&params[i])};
    }
    std::stable_sort(items.begin(), items.end(), [](const Item& a, const Item& b) {
        if (a.v != b.v) return a.v < b.v;
        return a.cost > b.cost;
    });
    std::vector<InstDesc> descs(count);
    cudaError_t e;
    void* buf = nullptr;
    const size_t bytes = sizeof(InstDesc) * (size_t)count + 2 * sizeof(double) * (size_t)count;
    if ((e = cudaMallocAsync(&buf, bytes, stream)) != cudaSuccess) return cuda_fail(e, "cudaMallocAsync");
    InstDesc* dd = reinterpret_cast<InstDesc*>(buf);
    double* pw = reinterpret_cast<double*>(reinterpret_cast<char*>(buf) + sizeof(InstDesc) * (size_t)count);
    for (int k = 0; k < count; ++k) {
        const int i = items[k].idx;
        InstDesc d = make_plain_desc(params[i], params[i].temp, params[i].temp);
        d.slot = i;
        d.pump_out = pump_out ? pump_out[i] : nullptr;
        d.signal_out = signal_out ? signal_out[i] : nullptr;
        d.power_out = pw + 2 * (size_t)i;
        descs[k] = d;
    }
    shg_status rc = SHG_OK;
    do {
        if ((e = cudaMemcpyAsync(dd, descs.data(), sizeof(InstDesc) * (size_t)count, cudaMemcpyHostToDevice,
                                 stream)) != cudaSuccess) {
            rc = cuda_fail(e, "cudaMemcpyAsync descs");
            break;
        }
        // groups: [begin, end) runs of the same variant, biggest total work first
        struct Group { const PlainVariant* v; int begin, end; double work; };
        std::vector<Group> groups;
        for (int k = 0; k < count;) {
            int j = k;
            double w = 0;
            while (j < count && items[j].v == items[k].v) w += items[j++].cost;
            groups.push_back({items[k].v, k, j, w});
            k = j;
        }
        std::sort(groups.begin(), groups.end(), [](const Group& a, const Group& b) { return a.work > b.work; });
        if (groups.size() == 1) {
            if ((e = groups[0].v->launch(dd + groups[0].begin, groups[0].end - groups[0].begin, stream)) != cudaSuccess) {
                rc = cuda_fail(e, "launch ssfm_plain_kernel");
                break;
            }
        } else {
            int dev = 0;
            cudaGetDevice(&dev);
            ForkStreams* f = nullptr;
            if ((e = fork_streams(dev, &f)) != cudaSuccess) { rc = cuda_fail(e, "stream pool"); break; }
            const int ng = (int)std::min<size_t>(groups.size(), ForkStreams::kMax);
            cudaEventRecord(f->ev[ForkStreams::kMax], stream);
            for (int g = 0; g < (int)groups.size(); ++g) {
                cudaStream_t s = f->s[g % ng];
                if (g < ng) cudaStreamWaitEvent(s, f->ev[ForkStreams::kMax], 0);
                if ((e = groups[g].v->launch(dd + groups[g].begin, groups[g].end - groups[g].begin, s)) != cudaSuccess) {
                    rc = cuda_fail(e, "launch ssfm_plain_kernel");
                    break;
                }
            }
            for (int g = 0; g < ng; ++g) {
                cudaEventRecord(f->ev[g], f->s[g]);
                cudaStreamWaitEvent(stream, f->ev[g], 0);
            }
            if (rc != SHG_OK) break;
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
        }
    } while (0);
    cudaFreeAsync(buf, stream);
    e = cudaGetLastError();
    if (rc == SHG_OK && e != cudaSuccess) rc = cuda_fail(e, "batch run");
    return rc;
}

}  // namespace shg
