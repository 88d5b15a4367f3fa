// Bloom pyramid, composite, tone map and pack (bloom.rs:28-125, renderer.rs:1116-1129), on the
// reference's layout: level 0 is the HDR image, levels 1..6 follow it in one float4 buffer.
// Each sum runs in the reference's order so the packed pixels match it bit for bit given the
// same HDR input.
#include "sr_kernels.h"

namespace srk {

Pyramid make_pyramid(uint32_t width, uint32_t height) {
    Pyramid p{};
    uint32_t w = width, h = height, off = 0;
    for (int k = 0; k <= SR_BLOOM_LEVELS; ++k) {
        p.w[k] = w;
        p.h[k] = h;
        p.off[k] = off;
        off += w * h;
        w = (w + 1) / 2;
        h = (h + 1) / 2;
    }
    p.off[SR_BLOOM_LEVELS + 1] = off;
    return p;
}

__constant__ float DOWN_W[4] = {0.125f, 0.375f, 0.375f, 0.125f};

// Level k from level k-1 with a [1 3 3 1]/8 filter per axis (bloom.rs:54-75).
__global__ void k_bloom_down(float4* pyr, Pyramid p, int k) {
    uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    uint32_t dw = p.w[k], dh = p.h[k];
    if (x >= dw || y >= dh) return;
    uint32_t sw = p.w[k - 1], sh = p.h[k - 1];
    const float4* src = pyr + p.off[k - 1];
    float ax = 0.0f, ay = 0.0f, az = 0.0f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        int syi = 2 * (int)y - 1 + j;
        syi = syi < 0 ? 0 : (syi > (int)sh - 1 ? (int)sh - 1 : syi);
        float rx = 0.0f, ry = 0.0f, rz = 0.0f;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            int sxi = 2 * (int)x - 1 + i;
            sxi = sxi < 0 ? 0 : (sxi > (int)sw - 1 ? (int)sw - 1 : sxi);
            float4 v = src[(size_t)syi * sw + sxi];
            rx = rx + v.x * DOWN_W[i];
            ry = ry + v.y * DOWN_W[i];
            rz = rz + v.z * DOWN_W[i];
        }
        ax = ax + rx * DOWN_W[j];
        ay = ay + ry * DOWN_W[j];
        az = az + rz * DOWN_W[j];
    }
    pyr[p.off[k] + (size_t)y * dw + x] = make_float4(ax, ay, az, 0.0f);
}

// upsample_at (bloom.rs:80-90): bilinear 2x of the coarse level at fine pixel (x, y).
__device__ __forceinline__ float4 upsample_at(const float4* c, uint32_t cw, uint32_t ch, uint32_t x, uint32_t y) {
    uint32_t mx = x / 2, my = y / 2;
    int ox = (x % 2 == 0) ? (int)mx - 1 : (int)mx + 1;
    int oy = (y % 2 == 0) ? (int)my - 1 : (int)my + 1;
    uint32_t x1 = (uint32_t)(ox < 0 ? 0 : (ox > (int)cw - 1 ? (int)cw - 1 : ox));
    uint32_t y1 = (uint32_t)(oy < 0 ? 0 : (oy > (int)ch - 1 ? (int)ch - 1 : oy));
    float4 a = c[(size_t)my * cw + mx], b = c[(size_t)my * cw + x1];
    float4 e = c[(size_t)y1 * cw + mx], g = c[(size_t)y1 * cw + x1];
    float r0x = a.x * 0.75f + b.x * 0.25f, r0y = a.y * 0.75f + b.y * 0.25f, r0z = a.z * 0.75f + b.z * 0.25f;
    float r1x = e.x * 0.75f + g.x * 0.25f, r1y = e.y * 0.75f + g.y * 0.25f, r1z = e.z * 0.75f + g.z * 0.25f;
    return make_float4(r0x * 0.75f + r1x * 0.25f, r0y * 0.75f + r1y * 0.25f, r0z * 0.75f + r1z * 0.25f, 0.0f);
}

// Level k += upsample(level k+1), coarsest first (bloom.rs:103-115).
__global__ void k_bloom_up(float4* pyr, Pyramid p, int k) {
    uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    uint32_t w = p.w[k], h = p.h[k];
    if (x >= w || y >= h) return;
    float4 up = upsample_at(pyr + p.off[k + 1], p.w[k + 1], p.h[k + 1], x, y);
    float4* dst = pyr + p.off[k] + (size_t)y * w + x;
    float4 v = *dst;
    *dst = make_float4(v.x + up.x, v.y + up.y, v.z + up.z, 0.0f);
}

// out = hdr * (1 - S) + up(level 1) * S / LEVELS, then pack_rgb_with_lut (bloom.rs:116-124,
// renderer.rs:1116-1129). The LUT is staged in shared memory.
__global__ void __launch_bounds__(256) k_bloom_composite(const float4* pyr, Pyramid p, uint32_t* rgb, const uint32_t* tables) {
    __shared__ uint8_t lut[SR_GAMMA_LUT_SIZE];
    for (uint32_t i = threadIdx.x + threadIdx.y * blockDim.x; i < SR_GAMMA_LUT_SIZE; i += blockDim.x * blockDim.y)
        lut[i] = (uint8_t)__ldg(tables + i);
    __syncthreads();
    uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= p.w[0] || y >= p.h[0]) return;
    const float strength = 0.04f;
    const float keep = 1.0f - strength;
    const float halo = strength / (float)SR_BLOOM_LEVELS;
    float4 up = upsample_at(pyr + p.off[1], p.w[1], p.h[1], x, y);
    float4 c = pyr[(size_t)y * p.w[0] + x];
    float cx = c.x * keep + up.x * halo, cy = c.y * keep + up.y * halo, cz = c.z * keep + up.z * halo;
    float mx = cx / (1.0f + cx * 0.35f), my = cy / (1.0f + cy * 0.35f), mz = cz / (1.0f + cz * 0.35f);
    mx = mx < 0.0f ? 0.0f : (mx > 1.0f ? 1.0f : mx);
    my = my < 0.0f ? 0.0f : (my > 1.0f ? 1.0f : my);
    mz = mz < 0.0f ? 0.0f : (mz > 1.0f ? 1.0f : mz);
    const float scale = (float)(SR_GAMMA_LUT_SIZE - 1);
    // `as usize` saturates: NaN and negatives to 0 (a clamped value is in [0, 1] unless NaN).
    float fx = mx * scale, fy = my * scale, fz = mz * scale;
    uint32_t ix = fx > 0.0f ? (uint32_t)fx : 0u, iy = fy > 0.0f ? (uint32_t)fy : 0u, iz = fz > 0.0f ? (uint32_t)fz : 0u;
    rgb[(size_t)y * p.w[0] + x] = ((uint32_t)lut[ix] << 16) | ((uint32_t)lut[iy] << 8) | (uint32_t)lut[iz];
}

cudaError_t launch_bloom(const FrameDev& f, const Pyramid& p, const uint32_t* tables, cudaStream_t st) {
    dim3 b(16, 16);
    for (int k = 1; k <= SR_BLOOM_LEVELS; ++k) {
        dim3 g((p.w[k] + 15) / 16, (p.h[k] + 15) / 16);
        k_bloom_down<<<g, b, 0, st>>>(f.hdr, p, k);
    }
    for (int k = SR_BLOOM_LEVELS - 1; k >= 1; --k) {
        dim3 g((p.w[k] + 15) / 16, (p.h[k] + 15) / 16);
        k_bloom_up<<<g, b, 0, st>>>(f.hdr, p, k);
    }
    dim3 g((p.w[0] + 15) / 16, (p.h[0] + 15) / 16);
    k_bloom_composite<<<g, b, 0, st>>>(f.hdr, p, f.rgb, tables);
    return cudaGetLastError();
}

}  // namespace srk
