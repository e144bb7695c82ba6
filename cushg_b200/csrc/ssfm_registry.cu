// ssfm_registry.cu — lookup of the compiled fused-march variants and the autotuner's
// choices (see ssfm_variants.h).
#include <mutex>
#include <vector>

#include "ssfm_variants.h"

namespace shg {

namespace {

std::mutex g_mu;
std::vector<const PlainVariant*> g_chosen;  // tuned variants, one per (precision, n, thermal)

template <typename F>
void for_each_variant(F&& f) {
    const VariantTable tables[] = {variants_f32_small(), variants_f32_128(), variants_f32_192(), variants_f32_256(),
                                   variants_f64_small(), variants_f64_large(), variants_thermal()};
    for (const VariantTable& t : tables)
        for (int i = 0; i < t.count; ++i)
            if (f(&t.v[i])) return;
}

}  // namespace

const PlainVariant* find_plain_variant(int precision, int n, int thermal) {
    const int th = thermal ? 1 : 0;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        for (const PlainVariant* v : g_chosen)
            if (v->precision == precision && v->n == n && v->thermal == th) return v;
    }
    const PlainVariant* found = nullptr;
    for_each_variant([&](const PlainVariant* v) {
        if (v->precision == precision && v->n == n && v->thermal == th) found = v;
        return found != nullptr;
    });
    return found;
}

int plain_candidates(int precision, int n, const PlainVariant** out, int max) {
    int k = 0;
    for_each_variant([&](const PlainVariant* v) {
        if (v->precision == precision && v->n == n && !v->thermal && k < max) out[k++] = v;
        return false;
    });
    return k;
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
