// ssfm_registry.cu — lookup of the compiled fused-march variants and the autotuner's
// choices (see ssfm_variants.h).
#include <mutex>
#include <vector>

#include "../../include/shg.h"
#include "ssfm_variants.h"

namespace shg {

namespace {

std::mutex g_mu;
std::vector<const PlainVariant*> g_chosen;  // tuned variants, one per (precision, n, thermal)

template <typename F>
void for_each_variant(F&& f) {
    const VariantTable tables[] = {variants_f32_small(), variants_f32_128(), variants_f32_192(), variants_f32_256(),
                                   variants_f64_small(), variants_f64_large(), variants_thermal(),
                                   variants_multipass()};
    for (const VariantTable& t : tables)
        for (int i = 0; i < t.count; ++i)
            if (f(&t.v[i])) return;
}

}  // namespace

const PlainVariant* find_plain_variant(int precision, int n, int thermal, int march) {
    const int th = thermal ? 1 : 0;
    if (march == SHG_MARCH_AUTO) {
        std::lock_guard<std::mutex> lk(g_mu);
        for (const PlainVariant* v : g_chosen)
            if (v->precision == precision && v->n == n && v->thermal == th) return v;
    }
    const PlainVariant *fused = nullptr, *multi = nullptr;
    for_each_variant([&](const PlainVariant* v) {
        if (v->precision == precision && v->n == n && v->thermal == th) {
            if (v->mp && !multi) multi = v;
            if (!v->mp && !fused) fused = v;
        }
        return false;
    });
    if (march == SHG_MARCH_FUSED) return fused;
    if (march == SHG_MARCH_MULTIPASS) return multi;
    // automatic: a thermal run marches on the multi-pass kernels where they are built.  One
    // thermal instance's fused cluster holds 1-16 SMs for every optical pass, which lies on the
    // run's critical path between two heat solves; the multi-pass launches spread each step
    // over the GPU (the optical passes of a 128 x 128 x 200 FP64 run: 47.6 -> 21.3 ms).  Plain runs, which
    // come in batches that fill the GPU with clusters, keep the fused march.
    if (th && multi) return multi;
    return fused ? fused : multi;
}

int plain_candidates(int precision, int n, const PlainVariant** out, int max) {
    int k = 0;
    for_each_variant([&](const PlainVariant* v) {
        if (v->precision == precision && v->n == n && !v->thermal && k < max) out[k++] = v;
        return false;
    });
    return k;
}

void clear_plain_choices() {
    std::lock_guard<std::mutex> lk(g_mu);
    g_chosen.clear();
}

void set_plain_choice(const PlainVariant* v) {
    std::lock_guard<std::mutex> lk(g_mu);
    for (const PlainVariant*& c : g_chosen)
        if (c->precision == v->precision && c->n == v->n && c->thermal == v->thermal) {
            c = v;
            return;
        }
    g_chosen.push_back(v);
}

}  // namespace shg
