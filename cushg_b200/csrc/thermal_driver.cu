// thermal_driver.cu — host driver of thermal runs: the -DTHERMAL outer optical-thermal
// loop of Solver::run (src/headers/Solver.h:321-373).
//
//   T = temp, oven faces = t_peltier, Q = 0                 (Solver.h:319-323)
//   repeat up to max_outer times:
//     Jacobi sweeps until the convergence value, taken on the first sweep of every
//     window of check_every sweeps, falls below tol; a value equal to the previous
//     check counts as converged                              (Solver.h:335-355)
//     (the checked sweep runs alone; the rest of the window runs jacobi_block sweeps
//     per launch through the temporally blocked kernel of jacobi_tb.cu)
//     Δk, n_p, n_s from T; pump, SH and propagators at T(NX/2, NY/2, 0)   (Solver.h:359-362)
//     one optical pass of nz steps that emits Q slice by slice (Solver.h:365, 300)
//     stop after a pass whose Jacobi loop converged at its first sweep (Solver.h:367)
//
// The host reads one scalar per check window; everything else stays on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <utility>
#include <vector>

#include "shg_host.h"
#include "ssfm_variants.h"
#include "thermal.h"

namespace shg {

namespace {

// Sweeps per launch: the caller's jacobi_block, else one.  On B200 the one-sweep kernel
// (one voxel per thread, neighbours through L1 / L2) measured faster than the blocked kernel
// at every depth and size tried, from L2-resident grids (128x128x200) to grids 20x the L2
// (512x512x250 FP64): 16.6 vs 28.9 us per sweep at 128x128x200 FP64, 325 vs 357 us at
// 512x512x250 FP64.  The blocked kernel is issue-bound (halo recomputation, one barrier per
// plane), not memory-bound.
int sweep_depth(const shg_params& p) {
    if (p.jacobi_block > 0) return p.jacobi_block;
    return 1;
}

// TMA maps of the two temperature buffers and Q for the blocked sweeps.
template <typename R>
struct SweepMaps {
    CUtensorMap a, b, q;
};

template <typename R>
shg_status make_sweep_maps(const R* Ta, const R* Tb, const R* Q, int n, int nz, SweepMaps<R>* m) {
    shg_status rc;
    if ((rc = make_tb_map<R>(Ta, n, nz, &m->a)) != SHG_OK) return rc;
    if ((rc = make_tb_map<R>(Tb, n, nz, &m->b)) != SHG_OK) return rc;
    return make_tb_map<R>(Q, n, nz, &m->q);
}

// `count` unchecked sweeps, `depth` per launch, ping-ponging cur / nxt (Ta and Tb of the
// maps); on return cur holds the latest temperature.
template <typename R>
cudaError_t run_sweeps(R*& cur, R*& nxt, const R* Ta, const SweepMaps<R>& m, const R* Q, const JacobiCoef<R>& k,
                       int boundary, int depth, int64_t count, unsigned* tb_err, cudaStream_t s) {
    while (count > 0) {
        const int t = (int)std::min<int64_t>(depth, count);
        cudaError_t e;
        if (t >= 2)
            e = launch_jacobi_tb<R>(cur == Ta ? m.a : m.b, m.q, nxt, k, boundary, t, tb_err, s);
        else
            e = launch_jacobi<R>(cur, nxt, Q, k, boundary, false, 0, nullptr, nullptr, s);
        if (e != cudaSuccess) return e;
        std::swap(cur, nxt);
        count -= t;
    }
    return cudaSuccess;
}

// One instance of a thermal run: its buffers, its Jacobi state and its latest optical pass.
template <typename R>
struct ThermalInst {
    const shg_params* p = nullptr;
    const void* signal_in = nullptr;
    void *pump_out = nullptr, *signal_out = nullptr, *slices_p = nullptr, *slices_s = nullptr;
    char* buf = nullptr;
    R *Ta = nullptr, *Tb = nullptr, *Q = nullptr, *DK = nullptr, *NP = nullptr, *NS = nullptr;
    double *partial = nullptr, *resid = nullptr, *power = nullptr;
    unsigned* tb_err = nullptr;
    R *cur = nullptr, *nxt = nullptr;  // cur holds the latest temperature (the reference's Tinic == Tfinal)
    SweepMaps<R> maps;
    JacobiCoef<R> k;
    double tol = 0.0;
    int check_every = 0, max_outer = 0, depth = 1;
    int64_t max_sweeps = 0;
    int64_t total = 0, counter = 0;  // sweeps of the run, of the current outer iteration
    int outer = 0;
    double last = 0.0, Tc = 0.0;
    double change = 0.0;  // heat_solver DIRECT: how far the latest solve moved T (the rule's measure)
    bool done = false;
    InstDesc d;  // descriptor of the latest optical pass
    double jacobi_ms = 0.0, optics_ms = 0.0;
    // Graphs of `count` one-sweep launches starting from Ta (parity 0) or Tb (parity 1): a
    // window of unchecked sweeps is a thousand launches of ~10 µs each, replayed from a graph
    // instead of being issued one by one.
    struct SweepGraph {
        int64_t count = 0;
        int parity = 0;
        cudaGraphExec_t exec = nullptr;
    };
    SweepGraph graphs[4];
};

// Windows shorter than this run as plain launches.
constexpr int64_t kSweepGraphMin = 64;

// `count` unchecked one-sweep launches of instance t from a graph (captured at first use for
// this start buffer and count, kept for the run): cur / nxt as run_sweeps leaves them.
template <typename R>
cudaError_t run_sweeps_graphed(ThermalInst<R>& t, int64_t count, cudaStream_t s) {
    const shg_params& p = *t.p;
    if (t.depth > 1 || count < kSweepGraphMin)
        return run_sweeps<R>(t.cur, t.nxt, t.Ta, t.maps, t.Q, t.k, p.boundary, t.depth, count, t.tb_err, s);
    const int parity = t.cur == t.Ta ? 0 : 1;
    typename ThermalInst<R>::SweepGraph* g = nullptr;
    for (auto& c : t.graphs)
        if (c.exec && c.count == count && c.parity == parity) g = &c;
    if (!g) {
        for (auto& c : t.graphs)
            if (!c.exec) {
                g = &c;
                break;
            }
        if (!g)  // every slot used by other counts: plain launches
            return run_sweeps<R>(t.cur, t.nxt, t.Ta, t.maps, t.Q, t.k, p.boundary, t.depth, count, t.tb_err, s);
        cudaStream_t cs = nullptr;
        cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
        if (e != cudaSuccess) return e;
        cudaGraph_t graph = nullptr;
        R* a = t.cur;
        R* b = t.nxt;
        e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            const cudaError_t el = run_sweeps<R>(a, b, t.Ta, t.maps, t.Q, t.k, p.boundary, 1, count, t.tb_err, cs);
            e = cudaStreamEndCapture(cs, &graph);
            if (el != cudaSuccess) e = el;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&g->exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        cudaStreamDestroy(cs);
        if (e != cudaSuccess) {
            g->exec = nullptr;
            return e;
        }
        g->count = count;
        g->parity = parity;
    }
    const cudaError_t e = cudaGraphLaunch(g->exec, s);
    if (e != cudaSuccess) return e;
    if (count & 1) std::swap(t.cur, t.nxt);
    return cudaSuccess;
}

template <typename R>
void ti_release(ThermalInst<R>& t) {
    for (auto& c : t.graphs)
        if (c.exec) {
            cudaGraphExecDestroy(c.exec);
            c.exec = nullptr;
        }
}

// Buffers of one instance.
template <typename R>
shg_status ti_alloc(ThermalInst<R>& t, cudaStream_t s) {
    const shg_params& p = *t.p;
    const int n = p.nx, nz = p.nz;
    const size_t nt = (size_t)n * n * nz, arr = sizeof(R) * nt;
    const size_t npart = jacobi_partials(p);
    const size_t bytes = 6 * arr + sizeof(double) * (npart + 4) + 256;
    cudaError_t e;
    if ((e = dev_alloc((void**)&t.buf, bytes, s)) != cudaSuccess) return cuda_fail(e, "cudaMallocAsync");
    t.Ta = reinterpret_cast<R*>(t.buf);
    t.Tb = t.Ta + nt;
    t.Q = t.Tb + nt;
    t.DK = t.Q + nt;
    t.NP = t.DK + nt;
    t.NS = t.NP + nt;
    t.partial = reinterpret_cast<double*>(t.NS + nt);
    t.resid = t.partial + npart;                            // [0] convergence value, [1] staging-error word
    t.power = t.resid + 2;                                  // [2]
    t.tb_err = reinterpret_cast<unsigned*>(t.resid + 1);    // set by a blocked sweep whose staging timed out
    t.k = make_jacobi_coef<R>(p);
    // Solver.h:332: tol = 5e-4 / TSIZE in the working precision
    t.tol = p.jacobi_tol > 0 ? p.jacobi_tol : (double)(R)(5e-4 / (double)nt);
    t.check_every = p.check_every > 0 ? p.check_every : 5000;
    t.max_sweeps = p.max_sweeps > 0 ? p.max_sweeps : ((int64_t)1 << 40);
    t.max_outer = p.max_outer > 0 ? p.max_outer : 20;
    t.depth = sweep_depth(p);
    t.cur = t.Ta;
    t.nxt = t.Tb;
    if (t.depth > 1) return make_sweep_maps<R>(t.Ta, t.Tb, t.Q, n, nz, &t.maps);
    return SHG_OK;
}

// Initial temperature of one instance (T = temp, oven faces = t_peltier, Q = 0, Solver.h:319-323).
template <typename R>
shg_status ti_init(ThermalInst<R>& t, cudaStream_t s) {
    cudaError_t e;
    if ((e = cudaMemsetAsync(t.resid, 0, 2 * sizeof(double), s)) != cudaSuccess) return cuda_fail(e, "memset");
    if ((e = launch_thermal_init<R>(t.Ta, t.Tb, t.Q, *t.p, s)) != cudaSuccess) return cuda_fail(e, "thermal init");
    return SHG_OK;
}

// The Jacobi loop of one outer iteration (Solver.h:335-355): the convergence value is taken on
// the first sweep of every window of check_every sweeps; a value equal to the previous check
// counts as converged; the rest of each window runs unchecked, `depth` sweeps per launch.
// FIXED rule: exactly max_sweeps sweeps, the last one reporting max |Tf - Ti|.
// DIRECT heat solver: the loop's fixed point in one solve, with the FP64 residual of one sweep
// of it (t.last) and how far it moved the temperature (t.change).
template <typename R>
shg_status ti_direct(ThermalInst<R>& t, HeatDirect* heat, cudaStream_t s) {
    const shg_params& p = *t.p;
    if (!heat) return fail(SHG_ERR_INVALID, "direct heat solve without a workspace");
    shg_status rc = heat->solve<R>(p, t.cur, t.Q, p.t_inf, s);
    if (rc != SHG_OK) return rc;
    double resid = 0.0, change = 0.0;
    const int rule = p.conv_rule == SHG_CONV_REFERENCE ? SHG_CONV_REFERENCE : SHG_CONV_MAXABS;
    if ((rc = heat->result(rule, &resid, &change, s)) != SHG_OK) return rc;
    if (!std::isfinite(resid) || !std::isfinite(change))
        return fail(SHG_ERR_NONFINITE, "heat solve: residual %g, change %g", resid, change);
    t.counter = 0;
    t.last = resid;
    t.change = change;
    return SHG_OK;
}

template <typename R>
shg_status ti_jacobi(ThermalInst<R>& t, HeatDirect* heat, cudaStream_t s) {
    const shg_params& p = *t.p;
    if (p.heat_solver == SHG_HEAT_DIRECT) return ti_direct<R>(t, heat, s);
    const size_t nt = (size_t)p.nx * p.nx * p.nz;
    cudaError_t e;
    double red = 1.0, aux = -1.0;
    int64_t counter = 0;
    // one checked sweep: its convergence value and the staging-error word
    auto checked = [&](int rule, double* out) -> shg_status {
        if ((e = launch_jacobi<R>(t.cur, t.nxt, t.Q, t.k, p.boundary, true, rule, t.partial, t.resid, s)) != cudaSuccess)
            return cuda_fail(e, "jacobi sweep");
        std::swap(t.cur, t.nxt);
        double h[2] = {0.0, 0.0};
        if ((e = cudaMemcpyAsync(h, t.resid, sizeof(h), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess)
            return cuda_fail(e, "jacobi residual");
        unsigned staged_err = 0;
        std::memcpy(&staged_err, &h[1], sizeof(staged_err));
        if (staged_err) return fail(SHG_ERR_CUDA, "blocked Jacobi sweep: a staged plane did not arrive");
        *out = h[0];
        return SHG_OK;
    };
    shg_status rc = SHG_OK;
    if (p.conv_rule == SHG_CONV_FIXED) {
        if ((e = run_sweeps_graphed<R>(t, t.max_sweeps - 1, s)) != cudaSuccess) return cuda_fail(e, "jacobi sweep");
        if ((rc = checked(SHG_CONV_MAXABS, &red)) != SHG_OK) return rc;
        counter = t.max_sweeps;
        if (!std::isfinite(red))
            return fail(SHG_ERR_NONFINITE, "Jacobi residual is %g after %lld sweeps", red, (long long)counter);
    }
    while (p.conv_rule != SHG_CONV_FIXED && red >= t.tol) {
        if (counter >= t.max_sweeps)
            return fail(SHG_ERR_NOT_CONVERGED, "Jacobi: %lld sweeps without reaching %g (last %g)", (long long)counter,
                        t.tol, red);
        double h0 = 0.0;
        if ((rc = checked(p.conv_rule, &h0)) != SHG_OK) return rc;
        if (counter > 0) aux = red;
        red = p.conv_rule == SHG_CONV_MAXABS ? h0 : (double)(R)(std::sqrt((R)h0) / (R)(double)nt);
        if (!std::isfinite(red))
            return fail(SHG_ERR_NONFINITE, "Jacobi residual is %g after %lld sweeps", red, (long long)counter);
        if (red == aux) red = 0.5 * t.tol;
        ++counter;
        if (red < t.tol) break;
        const int64_t left = std::min<int64_t>(t.check_every - 1, t.max_sweeps - counter);
        if ((e = run_sweeps_graphed<R>(t, left, s)) != cudaSuccess) return cuda_fail(e, "jacobi sweep");
        counter += std::max<int64_t>(left, 0);
    }
    t.counter = counter;
    t.total += counter;
    t.last = red;
    return SHG_OK;
}

// Δk, n_p, n_s from T and the descriptor of the optical pass from T(NX/2, NY/2, 0)
// (Solver.h:359-365), into t.d (host).
template <typename R>
shg_status ti_optics(ThermalInst<R>& t, cudaStream_t s) {
    const shg_params& p = *t.p;
    const int n = p.nx, nz = p.nz;
    cudaError_t e;
    if ((e = launch_optics<R>(t.cur, t.DK, t.NP, t.NS, p, s)) != cudaSuccess) return cuda_fail(e, "optics");
    R tc_h = 0;
    const size_t ic = (size_t)(n / 2) * n + n / 2;  // IDX(NX/2, NY/2, 0)
    if ((e = cudaMemcpyAsync(&tc_h, t.cur + ic, sizeof(R), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return cuda_fail(e, "read T");
    t.Tc = (double)tc_h;
    InstDesc d = make_plain_desc(p, t.Tc, t.Tc);
    const double dQ = 2.0 * p.deff / kPi, lp = p.lambda_p, ls = 0.5 * lp;
    d.kf_p = 1.0 * kPi * dQ / lp;
    d.kf_s = 0.5 * kPi * dQ / ls;
    d.bf_s = p.beta_s * 0.5 * kEps0 * kC;
    d.q_p = p.alpha_p * 0.5 * kC * kEps0;
    d.q_s = p.alpha_s * 0.5 * kC * kEps0;
    d.q_h = 0.5 * kC * kEps0;
    d.beta_s = p.beta_s;
    d.t_np = t.NP;
    d.t_ns = t.NS;
    d.t_dk = t.DK;
    d.t_q = t.Q;
    d.pw_s = d.pw_p = 0.5 * kEps0 * kC * d.dx * d.dy;
    d.signal_in = t.signal_in;
    d.has_signal_in = t.signal_in ? 1 : 0;
    d.pump_out = t.pump_out;
    d.signal_out = t.signal_out;
    d.power_out = t.power;
    d.slices_p = t.slices_p;
    d.slices_s = t.slices_s;
    d.nslices = (t.slices_p || t.slices_s) ? nz : 0;
    t.d = d;
    return SHG_OK;
}

// The thermal runs of `count` parameter sets (one grid side, precision and nz) in lockstep:
// each outer iteration runs every instance's Jacobi loop, then the optical passes of all
// instances still iterating as ONE launch sequence of the thermal march over them (a grid over
// the instances), then `hook` with their states.  An instance stops after its last pass
// (Solver.h:367, or max_outer); the others continue.  count == 1 is shg_solve's thermal run.
template <typename R>
shg_status thermal_batch_run(const shg_params* ps, int count, const void* const* signal_in, void* const* pump_out,
                             void* const* signal_out, void* const* temperature_out, shg_stats* stats, cudaStream_t s,
                             void* slices_p, void* slices_s, const ThermalBatchHook* hook) {
    const shg_params& p0 = ps[0];
    const PlainVariant* v = find_plain_variant(p0.precision, p0.nx, 1, p0.march);
    if (!v) return fail(SHG_ERR_UNSUPPORTED, "no thermal kernel for grid side %d", p0.nx);
    const size_t arr = sizeof(R) * (size_t)p0.nx * p0.nx * p0.nz;
    std::vector<ThermalInst<R>> ti(count);
    std::vector<InstDesc> hd(count);
    std::vector<ThermalState> states(count);
    std::vector<int> act(count);
    InstDesc* dd = nullptr;
    std::unique_ptr<HeatDirect> heat;  // one FP64 workspace for the batch's direct heat solves
    for (int i = 0; i < count; ++i)
        if (ps[i].heat_solver == SHG_HEAT_DIRECT && !heat) heat.reset(new HeatDirect);
    shg_status rc = SHG_OK;
    cudaError_t e;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    // per-phase timing: an instance's Jacobi loop between ej[0] and ej[1], the optics and the
    // batched optical pass between ej[1] and ej[2]
    cudaEvent_t ej[3] = {nullptr, nullptr, nullptr};
    for (auto& ev : ej) cudaEventCreate(&ev);
    do {
        if ((e = dev_alloc((void**)&dd, sizeof(InstDesc) * (size_t)count, s)) != cudaSuccess) {
            rc = cuda_fail(e, "cudaMallocAsync");
            break;
        }
        for (int i = 0; i < count && rc == SHG_OK; ++i) {
            ti[i].p = &ps[i];
            ti[i].signal_in = signal_in ? signal_in[i] : nullptr;
            ti[i].pump_out = pump_out ? pump_out[i] : nullptr;
            ti[i].signal_out = signal_out ? signal_out[i] : nullptr;
            ti[i].slices_p = slices_p;
            ti[i].slices_s = slices_s;
            rc = ti_alloc<R>(ti[i], s);
        }
        if (rc != SHG_OK) break;
        // the device time starts after the workspace is allocated (a pool that grows maps
        // memory on the host's time, while the stream idles)
        cudaEventRecord(t0, s);
        for (int i = 0; i < count && rc == SHG_OK; ++i) rc = ti_init<R>(ti[i], s);
        if (rc != SHG_OK) break;
        for (int g = 0; rc == SHG_OK; ++g) {
            int na = 0;
            for (int i = 0; i < count; ++i)
                if (!ti[i].done) act[na++] = i;
            if (na == 0) break;
            for (int a = 0; a < na && rc == SHG_OK; ++a) {
                ThermalInst<R>& t = ti[act[a]];
                cudaEventRecord(ej[0], s);
                if ((rc = ti_jacobi<R>(t, heat.get(), s)) != SHG_OK) break;
                cudaEventRecord(ej[1], s);
                if ((e = cudaEventSynchronize(ej[1])) != cudaSuccess) { rc = cuda_fail(e, "jacobi"); break; }
                float ms = 0.f;
                cudaEventElapsedTime(&ms, ej[0], ej[1]);
                t.jacobi_ms += ms;
            }
            if (rc != SHG_OK) break;
            cudaEventRecord(ej[1], s);
            for (int a = 0; a < na && rc == SHG_OK; ++a) {
                rc = ti_optics<R>(ti[act[a]], s);
                hd[a] = ti[act[a]].d;
            }
            if (rc != SHG_OK) break;
            if ((e = cudaMemcpyAsync(dd, hd.data(), sizeof(InstDesc) * (size_t)na, cudaMemcpyHostToDevice, s)) != cudaSuccess) {
                rc = cuda_fail(e, "descriptors");
                break;
            }
            if ((e = run_variant(v, dd, hd.data(), na, nullptr, s)) != cudaSuccess) { rc = cuda_fail(e, "thermal optical pass"); break; }
            cudaEventRecord(ej[2], s);
            if ((e = cudaEventSynchronize(ej[2])) != cudaSuccess) { rc = cuda_fail(e, "thermal optical pass"); break; }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ej[1], ej[2]);
            for (int a = 0; a < na; ++a) {
                ThermalInst<R>& t = ti[act[a]];
                ++t.outer;
                t.optics_ms += ms;
                // Solver.h:367: the last pass is the one whose Jacobi loop converged at its first
                // sweep; with the direct solver, the one whose solve moved T by less than tol
                const bool settled = t.p->heat_solver == SHG_HEAT_DIRECT ? t.change < t.tol : t.counter == 1;
                t.done = t.outer == t.max_outer || (t.p->conv_rule != SHG_CONV_FIXED && settled && g != 0);
                states[a] = {t.cur, t.NP, t.NS, t.DK, &hd[a], dd + a, t.counter, t.Tc, g, t.done, act[a], heat.get()};
            }
            if (hook && (rc = (*hook)(states.data(), na, s)) != SHG_OK) break;
        }
        if (rc != SHG_OK) break;
        for (int i = 0; i < count && rc == SHG_OK; ++i) {
            if (temperature_out && temperature_out[i] &&
                (e = cudaMemcpyAsync(temperature_out[i], ti[i].cur, arr, cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
                rc = cuda_fail(e, "temperature out");
        }
        if (rc != SHG_OK) break;
        cudaEventRecord(t1, s);
        if (stats) {
            std::vector<double> h(2 * (size_t)count);
            for (int i = 0; i < count && e == cudaSuccess; ++i)
                e = cudaMemcpyAsync(&h[2 * (size_t)i], ti[i].power, 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
            if (e != cudaSuccess || (e = cudaStreamSynchronize(s)) != cudaSuccess) {
                rc = cuda_fail(e, "thermal run");
                break;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, t0, t1);
            for (int i = 0; i < count; ++i) {
                shg_stats& st = stats[i];
                std::memset(&st, 0, sizeof(st));
                st.sh_power = h[2 * (size_t)i];
                st.pump_power = h[2 * (size_t)i + 1];
                st.jacobi_sweeps = ti[i].total;
                st.outer_iterations = ti[i].outer;
                st.steps = ps[i].nz;
                st.last_residual = ti[i].last;
                st.device_ms = ms;
                st.jacobi_ms = ti[i].jacobi_ms;
                st.optics_ms = ti[i].optics_ms;
                if (rc == SHG_OK && (!std::isfinite(st.sh_power) || !std::isfinite(st.pump_power)))
                    rc = count > 1 ? fail(SHG_ERR_NONFINITE, "instance %d: SH / pump power %g / %g", i, st.sh_power,
                                          st.pump_power)
                                   : fail(SHG_ERR_NONFINITE, "SH / pump power %g / %g", st.sh_power, st.pump_power);
            }
        }
    } while (0);
    cudaStreamSynchronize(s);  // the graphs' launches are done before their release
    if (heat) heat->release(s);
    for (auto& t : ti) {
        ti_release<R>(t);
        if (t.buf) cudaFreeAsync(t.buf, s);
    }
    if (dd) cudaFreeAsync(dd, s);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    for (cudaEvent_t ev : ej) cudaEventDestroy(ev);
    e = cudaGetLastError();
    if (rc == SHG_OK && e != cudaSuccess) rc = cuda_fail(e, "thermal run");
    return rc;
}

template <typename R>
shg_status heat_run(const shg_params& p, R* T, const R* Q, int64_t sweeps, cudaStream_t s) {
    const int n = p.nx, nz = p.nz;
    const size_t nt = (size_t)n * n * nz, arr = sizeof(R) * nt;
    // Q null (no heat source, the sweeps read none): one sweep per launch, whose kernels
    // take a null Q as zero
    const int depth = Q ? sweep_depth(p) : 1;
    cudaError_t e;
    char* buf = nullptr;
    if ((e = dev_alloc((void**)&buf, arr + 256, s)) != cudaSuccess) return cuda_fail(e, "cudaMallocAsync");
    R* other = reinterpret_cast<R*>(buf);
    unsigned* tb_err = reinterpret_cast<unsigned*>(buf + arr);
    shg_status rc = SHG_OK;
    do {
        SweepMaps<R> maps;
        if (depth > 1 && (rc = make_sweep_maps<R>(T, other, Q, n, nz, &maps)) != SHG_OK) break;
        // both buffers start alike, so the voxels no sweep writes (Dirichlet faces) agree
        if ((e = cudaMemcpyAsync(other, T, arr, cudaMemcpyDeviceToDevice, s)) != cudaSuccess ||
            (e = cudaMemsetAsync(tb_err, 0, sizeof(unsigned), s)) != cudaSuccess) {
            rc = cuda_fail(e, "heat sweeps set-up");
            break;
        }
        const JacobiCoef<R> k = make_jacobi_coef<R>(p);
        R* cur = T;
        R* nxt = other;
        if ((e = run_sweeps<R>(cur, nxt, T, maps, Q, k, p.boundary, depth, sweeps, tb_err, s)) != cudaSuccess) {
            rc = cuda_fail(e, "jacobi sweep");
            break;
        }
        if (cur != T && (e = cudaMemcpyAsync(T, cur, arr, cudaMemcpyDeviceToDevice, s)) != cudaSuccess) {
            rc = cuda_fail(e, "heat sweeps result");
            break;
        }
        unsigned h = 0;
        if ((e = cudaMemcpyAsync(&h, tb_err, sizeof(h), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess) {
            rc = cuda_fail(e, "heat sweeps");
            break;
        }
        if (h) rc = fail(SHG_ERR_CUDA, "blocked Jacobi sweep: a staged plane did not arrive");
    } while (0);
    cudaFreeAsync(buf, s);
    e = cudaGetLastError();
    if (rc == SHG_OK && e != cudaSuccess) rc = cuda_fail(e, "heat sweeps");
    return rc;
}

}  // namespace

shg_status heat_sweeps_device(const shg_params& p, void* temperature, const void* q, int64_t sweeps,
                              cudaStream_t stream) {
    if (p.precision == 32)
        return heat_run<float>(p, reinterpret_cast<float*>(temperature), reinterpret_cast<const float*>(q), sweeps, stream);
    return heat_run<double>(p, reinterpret_cast<double*>(temperature), reinterpret_cast<const double*>(q), sweeps, stream);
}

shg_status thermal_solve_device(const shg_params& p, const void* signal_in, void* pump_out, void* signal_out,
                                void* temperature_out, shg_stats* stats, cudaStream_t stream, void* slices_p,
                                void* slices_s, const ThermalHook* hook) {
    ThermalBatchHook bh;
    if (hook) bh = [hook](const ThermalState* st, int, cudaStream_t s) { return (*hook)(st[0], s); };
    return thermal_solve_batch(&p, 1, &signal_in, &pump_out, &signal_out, &temperature_out, stats, stream, slices_p,
                               slices_s, hook ? &bh : nullptr);
}

shg_status thermal_solve_batch(const shg_params* ps, int count, const void* const* signal_in, void* const* pump_out,
                               void* const* signal_out, void* const* temperature_out, shg_stats* stats,
                               cudaStream_t stream, void* slices_p, void* slices_s, const ThermalBatchHook* hook) {
    if (count <= 0) return SHG_OK;
    if (ps[0].precision == 32)
        return thermal_batch_run<float>(ps, count, signal_in, pump_out, signal_out, temperature_out, stats, stream,
                                        slices_p, slices_s, hook);
    return thermal_batch_run<double>(ps, count, signal_in, pump_out, signal_out, temperature_out, stats, stream,
                                     slices_p, slices_s, hook);
}

}  // namespace shg
