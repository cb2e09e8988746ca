// Autotuning of the kernel variants a context uses (no reference counterpart).
// ol_autotune measures the variants on a caller's document and keeps the
// fastest; the choice is recorded per device (name and SM count) in a plain
// text file, one line per device:
//   <device name>\t<SM count>\t<dict_slice>\t<dict_blocks_per_sm>\t<dict_heavy_divisor>\t<search_staged>
// and read back by ol_tuning_load (and by ol_ctx_create when OL_TUNING_FILE
// names such a file). Variants change speed only: every one computes the same
// results, which the tests check.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "runtime.h"

using namespace ol;

namespace {

bool valid(const ol_tuning &t) {
    return (t.dict_slice == 256 || t.dict_slice == 512 || t.dict_slice == 1024) && t.dict_blocks_per_sm <= 32 &&
           t.dict_heavy_divisor >= 1 && t.search_staged <= 1;
}

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

std::string device_key(const ol_ctx *ctx) {
    std::string name(ctx->name);
    for (char &c : name)
        if (c == '\t' || c == '\n') c = ' ';
    return name + "\t" + std::to_string(ctx->sm_count);
}

// Median of `reps` timed runs of fn (after one untimed run); fn returns false on error.
template <class F>
double time_median(int reps, F fn) {
    if (!fn()) return -1;
    std::vector<double> t;
    for (int i = 0; i < reps; i++) {
        double t0 = now_s();
        if (!fn()) return -1;
        t.push_back(now_s() - t0);
    }
    std::sort(t.begin(), t.end());
    return t[t.size() / 2];
}

}  // namespace

ol_status ol::load_tuning(ol_ctx *ctx, const char *path) {
    std::ifstream f(path);
    if (!f) return OL_ERR_NOT_FOUND;
    const std::string key = device_key(ctx);
    std::string line;
    bool found = false;
    ol_tuning t = ctx->tune;
    while (std::getline(f, line)) {
        if (line.compare(0, key.size(), key) != 0 || line.size() <= key.size() || line[key.size()] != '\t') continue;
        std::istringstream in(line.substr(key.size() + 1));
        ol_tuning r{};
        if (in >> r.dict_slice >> r.dict_blocks_per_sm >> r.dict_heavy_divisor >> r.search_staged && valid(r)) {
            t = r;
            found = true;
        }
    }
    if (!found) return OL_ERR_NOT_FOUND;
    ctx->tune = t;
    return OL_OK;
}

extern "C" ol_status ol_tuning_get(ol_ctx *ctx, ol_tuning *out) {
    if (!ctx || !out) return OL_ERR_INVALID_ARG;
    *out = ctx->tune;
    return OL_OK;
}

extern "C" ol_status ol_tuning_set(ol_ctx *ctx, const ol_tuning *t) {
    if (!ctx || !t) return OL_ERR_INVALID_ARG;
    if (!valid(*t)) return ctx_fail(ctx, OL_ERR_INVALID_ARG, "tuning values out of range");
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    ctx->tune = *t;
    return OL_OK;
}

extern "C" ol_status ol_tuning_load(ol_ctx *ctx, const char *path) {
    if (!ctx || !path) return OL_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    ol_status s = load_tuning(ctx, path);
    return s == OL_OK ? s : ctx_fail(ctx, s, std::string("no tuning for this device in ") + path);
}

extern "C" ol_status ol_autotune(ol_ctx *ctx, const ol_doc *d, const ol_patset *set, const uint8_t *const *patterns,
                                 const uint32_t *lens, uint32_t n, const char *path, ol_tuning *out) {
    if (!ctx || !d || (n && (!patterns || !lens))) return OL_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    const ol_tuning keep = ctx->tune;
    ol_tuning best = keep;
    cudaStream_t st = ctx->stream;

    // Dictionary: slice and resident blocks, then the heavy threshold. Timed
    // without emitting the hits, which every variant writes the same way.
    if (set && d->text_len) {
        std::vector<uint32_t> counts(ol_patset_len(set));
        uint64_t total = 0;
        auto run = [&]() {
            return many_run(ctx, d, set, 0, 0, counts.data(), &total, HitDest{}, nullptr, nullptr, 0) == OL_OK;
        };
        double best_t = 1e30;
        for (uint32_t slice : {256u, 512u, 1024u})
            for (uint32_t bps : {0u, 2u, 3u, 4u}) {
                ctx->tune = best;
                ctx->tune.dict_slice = slice;
                ctx->tune.dict_blocks_per_sm = bps;
                double t = time_median(2, run);
                if (t >= 0 && t < best_t) {
                    best_t = t;
                    best.dict_slice = slice;
                    best.dict_blocks_per_sm = bps;
                }
            }
        for (uint32_t div : {128u, 512u, 2048u}) {
            ctx->tune = best;
            ctx->tune.dict_heavy_divisor = div;
            double t = time_median(2, run);
            if (t >= 0 && t < best_t) {
                best_t = t;
                best.dict_heavy_divisor = div;
            }
        }
    }

    // Substring search: staged or recomputing, with every hit written.
    if (n && d->text_len) {
        std::vector<const uint8_t *> p2;
        std::vector<uint32_t> l2;
        for (uint32_t i = 0; i < n; i++)
            if (lens[i] && lens[i] <= d->text_len) {
                p2.push_back(patterns[i]);
                l2.push_back(lens[i]);
            }
        const uint32_t m = (uint32_t)p2.size();
        if (m) {
            // exact totals first (count only), then room for every hit
            std::vector<uint32_t> tot(m), zero(m, 0);
            ctx->tune = best;
            DevBuf outs;
            cudaError_t e = outs.reserve(((size_t)m + 64) * 4, st);
            std::vector<uint32_t *> o0(m, (uint32_t *)outs.ptr + 64);
            ol_status s = e == cudaSuccess ? OL_OK : ctx_cuda(ctx, e, "autotune");
            if (s == OL_OK)
                s = ol_search_multi_async(ctx, d, p2.data(), l2.data(), m, zero.data(), (uint32_t *)outs.ptr, o0.data());
            if (s == OL_OK && cudaMemcpyAsync(tot.data(), outs.ptr, (size_t)m * 4, cudaMemcpyDeviceToHost, st) == cudaSuccess &&
                cudaStreamSynchronize(st) == cudaSuccess) {
                size_t words = 64;
                for (uint32_t x : tot) words += std::max<uint32_t>(x, 1);
                outs.release(st);
                if ((e = outs.reserve(words * 4, st)) == cudaSuccess) {
                    std::vector<uint32_t *> o(m);
                    size_t w = 64;
                    for (uint32_t i = 0; i < m; i++) {
                        o[i] = (uint32_t *)outs.ptr + w;
                        w += std::max<uint32_t>(tot[i], 1);
                    }
                    double best_t = 1e30;
                    for (uint32_t staged : {1u, 0u}) {
                        ctx->tune = best;
                        ctx->tune.search_staged = staged;
                        double t = time_median(3, [&]() {
                            return ol_search_multi_async(ctx, d, p2.data(), l2.data(), m, tot.data(),
                                                         (uint32_t *)outs.ptr, o.data()) == OL_OK &&
                                   cudaStreamSynchronize(st) == cudaSuccess;
                        });
                        if (t >= 0 && t < best_t) {
                            best_t = t;
                            best.search_staged = staged;
                        }
                    }
                }
            }
            outs.release(st);
            cudaStreamSynchronize(st);
        }
    }
    ctx->tune = best;
    if (out) *out = best;

    if (path) {
        // replace this device's line, keep the others
        const std::string key = device_key(ctx);
        std::vector<std::string> lines;
        {
            std::ifstream f(path);
            std::string line;
            while (std::getline(f, line))
                if (!line.empty() && !(line.compare(0, key.size(), key) == 0 && line.size() > key.size() &&
                                       line[key.size()] == '\t'))
                    lines.push_back(line);
        }
        std::ostringstream l;
        l << key << "\t" << best.dict_slice << "\t" << best.dict_blocks_per_sm << "\t" << best.dict_heavy_divisor << "\t"
          << best.search_staged;
        lines.push_back(l.str());
        std::ofstream f(path, std::ios::trunc);
        if (!f) return ctx_fail(ctx, OL_ERR_INVALID_ARG, std::string("cannot write ") + path);
        for (auto &x : lines) f << x << "\n";
    }
    return OL_OK;
}
