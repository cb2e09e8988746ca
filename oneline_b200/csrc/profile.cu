// Opt-in profiling of a context: GPU pass durations from CUDA events on the
// context's stream, plus host step marks. Replaces the reference's StageTimer
// (crates/oneline-gpu/src/timing.rs:16-107, wgpu timestamp queries around each
// compute pass and host marks) and fills an ol_profile like its Profile
// (timing.rs:109-124). Calls made while no profile is open pay one pointer
// test per pass.
#include <cuda_runtime.h>

#include <chrono>
#include <cstring>
#include <string>
#include <vector>

#include "runtime.h"

namespace ol {

struct ProfPass {
    const char *label;
    cudaEvent_t start, end;
};

struct Prof {
    std::chrono::steady_clock::time_point first, last;
    std::vector<std::pair<const char *, uint64_t>> host_steps;
    std::vector<ProfPass> passes;
};

namespace {
uint64_t ns_between(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(b - a).count();
}

bool capturing(cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    return cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone;
}

void copy_label(char *dst, const char *src) {
    strncpy(dst, src, OL_PROFILE_LABEL_LEN - 1);
    dst[OL_PROFILE_LABEL_LEN - 1] = 0;
}

void release(Prof *p) {
    for (auto &x : p->passes) {
        if (x.start) cudaEventDestroy(x.start);
        if (x.end) cudaEventDestroy(x.end);
    }
    delete p;
}
}  // namespace

GpuPass::GpuPass(ol_ctx *c, const char *label, cudaStream_t on) : ctx(c), stream(on ? on : (c ? c->stream : nullptr)) {
    Prof *p = c ? c->prof : nullptr;
    if (!p || p->passes.size() >= OL_PROFILE_MAX_STEPS || capturing(stream)) return;
    ProfPass x{label, nullptr, nullptr};
    if (cudaEventCreate(&x.start) != cudaSuccess || cudaEventCreate(&x.end) != cudaSuccess ||
        cudaEventRecord(x.start, stream) != cudaSuccess) {
        if (x.start) cudaEventDestroy(x.start);
        if (x.end) cudaEventDestroy(x.end);
        cudaGetLastError();
        return;
    }
    p->passes.push_back(x);
    index = (int)p->passes.size() - 1;
}

void GpuPass::done() {
    if (index < 0 || !ctx->prof || index >= (int)ctx->prof->passes.size()) return;
    if (cudaEventRecord(ctx->prof->passes[index].end, stream) != cudaSuccess) cudaGetLastError();
    index = -1;
}

void prof_mark(ol_ctx *ctx, const char *label) {
    Prof *p = ctx ? ctx->prof : nullptr;
    if (!p || p->host_steps.size() >= OL_PROFILE_MAX_STEPS) return;
    auto now = std::chrono::steady_clock::now();
    p->host_steps.emplace_back(label, ns_between(p->last, now));
    p->last = now;
}

void prof_discard(ol_ctx *ctx) {
    if (ctx && ctx->prof) {
        release(ctx->prof);
        ctx->prof = nullptr;
    }
}

}  // namespace ol

using namespace ol;

extern "C" ol_status ol_profile_begin(ol_ctx *ctx) {
    if (!ctx) return OL_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    prof_discard(ctx);
    ctx->prof = new Prof();
    ctx->prof->first = ctx->prof->last = std::chrono::steady_clock::now();
    return OL_OK;
}

extern "C" ol_status ol_profile_end(ol_ctx *ctx, ol_profile *out) {
    if (!ctx || !out) return OL_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    Prof *p = ctx->prof;
    if (!p) return ctx_fail(ctx, OL_ERR_INVALID_ARG, "no profile is open on this context (ol_profile_begin)");
    cudaSetDevice(ctx->device);
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    memset(out, 0, sizeof *out);
    out->wall_ns = ns_between(p->first, p->last);
    for (auto &h : p->host_steps) {
        ol_profile_step &s = out->host_steps[out->n_host_steps++];
        copy_label(s.label, h.first);
        s.ns = h.second;
    }
    uint64_t total = 0;
    for (auto &x : p->passes) {
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, x.start, x.end);
        ol_profile_step &s = out->gpu_passes[out->n_gpu_passes++];
        copy_label(s.label, x.label);
        s.ns = (uint64_t)((double)ms * 1e6);
        total += s.ns;
    }
    out->gpu_total_ns = total;
    ctx->prof = nullptr;
    release(p);
    return ctx_cuda(ctx, e, "profile");
}
