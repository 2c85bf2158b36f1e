// After the gather (scope row f3): progressive accumulation of the output planes and their
// normalisation by the number of light paths (Renderer::Add / Normalize, Render.cpp:298-316,
// 639-664), the image error against a reference image (CReferenceImage::GetError,
// CReferenceImage.cpp:28-51), and PFM / Radiance HDR export (CExport::ExportPFM / ExportHDR,
// Utils/CExport.cpp:22-106).
//
// The reference blends frames into RGBA32F targets and normalises in a shader, all in FP32; the
// sums here are FP64 (a long accumulation in FP32 loses the late frames' low bits), and the
// normalised planes are rounded to float once.  The error sums the clamped squared differences in
// FP64 in a fixed order (the reference sums in FP32 in pixel order).
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "arc_internal.h"

namespace arc {
namespace {

constexpr int kPostThreads = 256;

struct AccumArgs {
    const float4* plane[3];  // result, radiance, antiradiance (NULL: skipped)
    int64_t opitch;
    double* sum;             // [pixel][9]
    int64_t apitch;
    int width, height;
};

__global__ void __launch_bounds__(kPostThreads) accumulate_kernel(AccumArgs a) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)a.width * a.height) return;
    const int x = (int)(i % a.width), y = (int)(i / a.width);
    double* s = a.sum + 9 * ((int64_t)y * a.apitch + x);
#pragma unroll
    for (int p = 0; p < 3; ++p) {
        if (!a.plane[p]) continue;
        const float4 v = a.plane[p][(int64_t)y * a.opitch + x];
        s[3 * p + 0] += (double)v.x;
        s[3 * p + 1] += (double)v.y;
        s[3 * p + 2] += (double)v.z;
    }
}

struct NormArgs {
    const double* sum;
    int64_t apitch;
    double inv;              // 1 / paths (0 for none, as Normalize)
    float4* plane[3];
    double* result64;
    int64_t opitch;
    int width, height;
};

__global__ void __launch_bounds__(kPostThreads) normalize_kernel(NormArgs a) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)a.width * a.height) return;
    const int x = (int)(i % a.width), y = (int)(i / a.width);
    const double* s = a.sum + 9 * ((int64_t)y * a.apitch + x);
    const int64_t o = (int64_t)y * a.opitch + x;
#pragma unroll
    for (int p = 0; p < 3; ++p) {
        if (!a.plane[p]) continue;
        a.plane[p][o] = make_float4((float)(s[3 * p] * a.inv), (float)(s[3 * p + 1] * a.inv),
                                    (float)(s[3 * p + 2] * a.inv), 1.0f);
    }
    if (a.result64)
        for (int c = 0; c < 3; ++c) a.result64[3 * o + c] = s[c] * a.inv;
}

// Per block: sums over its pixels of min(100, d^2) per channel, d = reference - image in FP32 as
// GetError computes it; block partials in FP64, combined in block order by error_finish.
__global__ void __launch_bounds__(kPostThreads) error_partials(const float4* ref, const float4* img, int width,
                                                              int height, int64_t pitch, double* partial) {
    __shared__ double red[3][kPostThreads / 32];
    const int64_t n = (int64_t)width * height;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % width), y = (int)(i / width);
        const float4 v = ref[(int64_t)y * pitch + x], u = img[(int64_t)y * pitch + x];
        const float d[3] = {v.x - u.x, v.y - u.y, v.z - u.z};
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[c] += (double)fminf(100.0f, d[c] * d[c]);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double v = acc[c];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[c][w] = v;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double v = 0.0;
        for (int k = 0; k < kPostThreads / 32; ++k) v += red[threadIdx.x][k];
        partial[3 * blockIdx.x + threadIdx.x] = v;
    }
}

__global__ void error_finish(const double* partial, int blocks, double* out) {
    if (threadIdx.x >= 3) return;
    double v = 0.0;
    for (int b = 0; b < blocks; ++b) v += partial[3 * b + threadIdx.x];
    out[threadIdx.x] = v;
}

// Radiance RGBE of one pixel (Ward, "Real Pixels", Graphics Gems II, 1991).
void rgbe(float r, float g, float b, unsigned char* e) {
    const float v = std::fmax(r, std::fmax(g, b));
    if (!(v >= 1e-32f)) {  // also NaN
        e[0] = e[1] = e[2] = e[3] = 0;
        return;
    }
    int ex;
    const float m = std::frexp(v, &ex) * 256.0f / v;
    e[0] = (unsigned char)std::fmax(0.0f, r * m);
    e[1] = (unsigned char)std::fmax(0.0f, g * m);
    e[2] = (unsigned char)std::fmax(0.0f, b * m);
    e[3] = (unsigned char)(ex + 128);
}

}  // namespace
}  // namespace arc

using namespace arc;

extern "C" arc_status arc_accumulate(arc_context* ctx, const ArcOutputView* frame, const ArcAccumView* acc) {
    ARC_CHECK_ARG(ctx && frame && acc && acc->sum, "NULL argument");
    ARC_CHECK_ARG(acc->width > 0 && acc->height > 0 && acc->pitch >= acc->width && frame->pitch >= acc->width,
                  "bad accumulation view");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    AccumArgs a;
    a.plane[0] = reinterpret_cast<const float4*>(frame->result);
    a.plane[1] = reinterpret_cast<const float4*>(frame->radiance);
    a.plane[2] = reinterpret_cast<const float4*>(frame->antiradiance);
    a.opitch = frame->pitch;
    a.sum = acc->sum;
    a.apitch = acc->pitch;
    a.width = acc->width;
    a.height = acc->height;
    const int64_t px = (int64_t)acc->width * acc->height;
    stage_begin(ctx, "accumulate");
    accumulate_kernel<<<(unsigned)((px + kPostThreads - 1) / kPostThreads), kPostThreads, 0, ctx->stream>>>(a);
    stage_end(ctx, 1);
    ARC_TRY_CUDA(cudaGetLastError());
    return ARC_OK;
}

extern "C" arc_status arc_accum_clear(arc_context* ctx, const ArcAccumView* acc) {
    ARC_CHECK_ARG(ctx && acc && acc->sum && acc->height > 0 && acc->pitch > 0, "NULL argument");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    ARC_TRY_CUDA(cudaMemsetAsync(acc->sum, 0, (size_t)acc->height * acc->pitch * 9 * sizeof(double), ctx->stream));
    return ARC_OK;
}

extern "C" arc_status arc_accum_normalize(arc_context* ctx, const ArcAccumView* acc, int64_t num_paths,
                                          const ArcOutputView* out) {
    ARC_CHECK_ARG(ctx && acc && acc->sum && out, "NULL argument");
    ARC_CHECK_ARG(num_paths >= 0, "negative path count");
    ARC_CHECK_ARG(acc->width > 0 && acc->height > 0 && acc->pitch >= acc->width && out->pitch >= acc->width,
                  "bad accumulation view");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    NormArgs a;
    a.sum = acc->sum;
    a.apitch = acc->pitch;
    a.inv = num_paths > 0 ? 1.0 / (double)num_paths : 0.0;
    a.plane[0] = reinterpret_cast<float4*>(out->result);
    a.plane[1] = reinterpret_cast<float4*>(out->radiance);
    a.plane[2] = reinterpret_cast<float4*>(out->antiradiance);
    a.result64 = out->result_fp64;
    a.opitch = out->pitch;
    a.width = acc->width;
    a.height = acc->height;
    const int64_t px = (int64_t)acc->width * acc->height;
    stage_begin(ctx, "normalize");
    normalize_kernel<<<(unsigned)((px + kPostThreads - 1) / kPostThreads), kPostThreads, 0, ctx->stream>>>(a);
    stage_end(ctx, 1);
    ARC_TRY_CUDA(cudaGetLastError());
    return ARC_OK;
}

extern "C" arc_status arc_image_error(arc_context* ctx, const float* reference, const float* image, int32_t width,
                                      int32_t height, int64_t pitch, int32_t metric, double* error,
                                      double* channel_rmse) {
    ARC_CHECK_ARG(ctx && reference && image && error, "NULL argument");
    ARC_CHECK_ARG(width > 0 && height > 0 && pitch >= width, "bad image size");
    ARC_CHECK_ARG(metric == ARC_ERROR_REFERENCE || metric == ARC_ERROR_RMSE, "unknown error metric");
    ARC_TRY_CUDA(cudaSetDevice(ctx->device));
    const int blocks = std::min<int64_t>(4 * ctx->sm_count, ((int64_t)width * height + kPostThreads - 1) / kPostThreads);
    double* partial = nullptr;
    ARC_TRY(ctx->arena.get("error_partials", (size_t)(3 * blocks + 3) * sizeof(double),
                           reinterpret_cast<void**>(&partial)));
    stage_begin(ctx, "image_error");
    error_partials<<<blocks, kPostThreads, 0, ctx->stream>>>(reinterpret_cast<const float4*>(reference),
                                                             reinterpret_cast<const float4*>(image), width, height,
                                                             pitch, partial);
    error_finish<<<1, 32, 0, ctx->stream>>>(partial, blocks, partial + 3 * blocks);
    stage_end(ctx, 2);
    ARC_TRY_CUDA(cudaGetLastError());
    double s[3];
    ARC_TRY_CUDA(cudaMemcpyAsync(s, partial + 3 * blocks, sizeof(s), cudaMemcpyDeviceToHost, ctx->stream));
    ARC_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    double e[3];
    for (int c = 0; c < 3; ++c) e[c] = std::sqrt(s[c] / ((double)width * height));
    if (channel_rmse)
        for (int c = 0; c < 3; ++c) channel_rmse[c] = e[c];
    // GetError returns 1/3 (e.x * e.y + e.z) (CReferenceImage.cpp:50); the mean is meant
    *error = metric == ARC_ERROR_REFERENCE ? (e[0] * e[1] + e[2]) / 3.0 : (e[0] + e[1] + e[2]) / 3.0;
    return ARC_OK;
}

namespace {

// ARC_ERR_IO with the failing step, the path and the C library's reason as the thread's message
arc_status io_error(const char* what, const char* path) {
    arc::set_last_error(std::string(what) + " " + path + ": " + std::strerror(errno));
    return ARC_ERR_IO;
}

}  // namespace

extern "C" arc_status arc_export_pfm(const char* path, const float* rgba, int32_t width, int32_t height,
                                     int64_t pitch) {
    ARC_CHECK_ARG(path && rgba && width > 0 && height > 0 && pitch >= width, "bad argument");
    FILE* f = std::fopen(path, "wb");
    if (!f) return io_error("arc_export_pfm: cannot open", path);
    // little-endian (scale -1), rows bottom to top; this plane's row 0 is the top of the image
    std::fprintf(f, "PF\n%d %d\n-1.0\n", width, height);
    std::vector<float> row(3 * (size_t)width);
    bool ok = true;
    for (int y = height - 1; y >= 0 && ok; --y) {
        const float* src = rgba + 4 * (size_t)y * pitch;
        for (int x = 0; x < width; ++x)
            for (int c = 0; c < 3; ++c) row[3 * x + c] = src[4 * x + c];
        ok = std::fwrite(row.data(), sizeof(float), row.size(), f) == row.size();
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? ARC_OK : io_error("export: cannot write", path);
}

extern "C" arc_status arc_export_hdr(const char* path, const float* rgba, int32_t width, int32_t height,
                                     int64_t pitch) {
    ARC_CHECK_ARG(path && rgba && width > 0 && height > 0 && pitch >= width, "bad argument");
    FILE* f = std::fopen(path, "wb");
    if (!f) return io_error("arc_export_hdr: cannot open", path);
    std::fprintf(f, "#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y %d +X %d\n", height, width);
    std::vector<unsigned char> px(4 * (size_t)width), out;
    const bool rle = width >= 8 && width <= 0x7fff;  // the run-length scanline format's range
    bool ok = true;
    for (int y = 0; y < height && ok; ++y) {
        const float* src = rgba + 4 * (size_t)y * pitch;
        for (int x = 0; x < width; ++x) rgbe(src[4 * x], src[4 * x + 1], src[4 * x + 2], &px[4 * x]);
        out.clear();
        if (rle) {
            // scanline marker, then each component as literal packets of at most 128 bytes
            out.push_back(2);
            out.push_back(2);
            out.push_back((unsigned char)(width >> 8));
            out.push_back((unsigned char)(width & 0xff));
            for (int c = 0; c < 4; ++c)
                for (int x0 = 0; x0 < width; x0 += 128) {
                    const int n = std::min(128, width - x0);
                    out.push_back((unsigned char)n);
                    for (int x = x0; x < x0 + n; ++x) out.push_back(px[4 * x + c]);
                }
        } else {
            out.assign(px.begin(), px.end());
        }
        ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? ARC_OK : io_error("export: cannot write", path);
}
