// Property check of the fold's host-side chunking (fold.cu: fold_chunks and
// fold_chunk_list, C++ functions the library exports beside its C ABI) on
// seeded sorted time series with gaps: the bounded list equals the chunking
// into a buffer of n + 2 offsets; the chunks tile [0, n); each holds at most
// chunk_cap observations and spans at most min(nb, span_cap) - 2 cells at
// scale_max (so its cells are distinct bins); each but the last ends only
// where the next observation would break one of those limits. Prints one
// JSON line of counts.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

namespace fbls {
int fold_chunks(const double* time, int n, double scale_max, int nb, int span_cap, int chunk_cap, int* out,
                int capacity);
int fold_chunk_list(const double* time, int n, double scale_max, int nb, int span_cap, int chunk_cap,
                    std::vector<int>& out);
}  // namespace fbls

int main() {
    std::mt19937_64 rng(20261204);
    auto uni = [&](double a, double b) { return std::uniform_real_distribution<double>(a, b)(rng); };
    int cases = 0, bad_equal = 0, bad_cover = 0, bad_limits = 0, bad_ends = 0;
    double offsets = 0.0, bound = 0.0, full_size = 0.0;
    for (int it = 0; it < 2000; it++) {
        const int n = 1 + (int)(rng() % 30000);
        std::vector<double> t(n);
        double x = uni(0.0, 5.0);
        const double step = std::exp(uni(std::log(1e-4), std::log(0.05)));
        for (int i = 0; i < n; i++) {
            x += (rng() % 50 == 0) ? step * (double)(1 + rng() % 2000) : step * uni(0.0, 2.0);
            t[i] = x;
        }
        const int nb = 8 + (int)(rng() % 4000);
        const double scale_max = nb / std::exp(uni(std::log(0.3), std::log(30.0)));
        const int span_cap = (rng() % 2) ? nb : 8 + (int)(rng() % 4000);
        const int chunk_cap = (rng() % 2) ? 2048 : 1 + (int)(rng() % 3000);
        std::vector<int> full((size_t)n + 2);
        const int cf = fbls::fold_chunks(t.data(), n, scale_max, nb, span_cap, chunk_cap, full.data(), n + 2);
        std::vector<int> list;
        const int cl = fbls::fold_chunk_list(t.data(), n, scale_max, nb, span_cap, chunk_cap, list);
        cases++;
        if (cf != cl || (int)list.size() != cl + 1 || !std::equal(list.begin(), list.end(), full.begin())) {
            bad_equal++;
            continue;
        }
        offsets += (double)list.size();
        bound += (double)list.capacity();
        full_size += (double)n + 2.0;
        bool cover = list[0] == 0 && list[cl] == n;
        for (int c = 0; c < cl; c++) cover = cover && list[c + 1] > list[c];
        if (!cover) {
            bad_cover++;
            continue;
        }
        const int cells = std::min(nb, span_cap) - 4;
        const double span = (double)std::max(cells, 1) / scale_max;
        for (int c = 0; c < cl; c++) {
            const int b = list[c], e = list[c + 1];
            const double spanned = std::floor(t[e - 1] * scale_max) - std::floor(t[b] * scale_max) + 1.0;
            if (e - b > chunk_cap || spanned > (double)(std::min(nb, span_cap) - 2)) bad_limits++;
            if (c + 1 < cl && e - b < chunk_cap && !(t[e] >= t[b] + span)) bad_ends++;
        }
    }
    std::printf("{\"cases\": %d, \"bad_equal\": %d, \"bad_cover\": %d, \"bad_limits\": %d, \"bad_ends\": %d, "
                "\"bound_over_offsets\": %.3f, \"bound_over_full\": %.4f}\n",
                cases, bad_equal, bad_cover, bad_limits, bad_ends, bound / offsets, bound / full_size);
    return 0;
}
