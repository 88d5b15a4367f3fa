// Bloom over the pyramids of every observer of a batch, one launch per level (included by
// sr_fast.cu, which defines find_obs and ObsDev).
#pragma once

namespace srk {

// Bloom over every observer's pyramid (bloom.rs:54-125); `pre` is the per-observer prefix of the
// level's pixel counts.
__constant__ float DOWN_WB[4] = {0.125f, 0.375f, 0.375f, 0.125f};

__global__ void k_bloom_down_batch(float4* hdr, const ObsDev* obs, const uint32_t* pre, uint32_t n, int k) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= __ldg(pre + n)) return;
    uint32_t o = find_obs(pre, n, i);
    const ObsDev& od = obs[o];
    uint32_t l = i - __ldg(pre + o);
    uint32_t dw = od.lw[k], x = l % dw, y = l / dw;
    uint32_t sw = od.lw[k - 1], sh = od.lh[k - 1];
    const float4* src = hdr + od.pyr_base + od.loff[k - 1];
    float ax = 0.0f, ay = 0.0f, az = 0.0f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        int syi = 2 * (int)y - 1 + j;
        syi = syi < 0 ? 0 : (syi > (int)sh - 1 ? (int)sh - 1 : syi);
        float rx = 0.0f, ry = 0.0f, rz = 0.0f;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            int sxi = 2 * (int)x - 1 + q;
            sxi = sxi < 0 ? 0 : (sxi > (int)sw - 1 ? (int)sw - 1 : sxi);
            float4 v = src[(size_t)syi * sw + sxi];
            rx = rx + v.x * DOWN_WB[q];
            ry = ry + v.y * DOWN_WB[q];
            rz = rz + v.z * DOWN_WB[q];
        }
        ax = ax + rx * DOWN_WB[j];
        ay = ay + ry * DOWN_WB[j];
        az = az + rz * DOWN_WB[j];
    }
    hdr[od.pyr_base + od.loff[k] + l] = make_float4(ax, ay, az, 0.0f);
}

__device__ __forceinline__ float4 upsample_b(const float4* c, uint32_t cw, uint32_t ch, uint32_t x, uint32_t y) {
    uint32_t mx = x / 2, my = y / 2;
    int ox = (x % 2 == 0) ? (int)mx - 1 : (int)mx + 1;
    int oy = (y % 2 == 0) ? (int)my - 1 : (int)my + 1;
    uint32_t x1 = (uint32_t)(ox < 0 ? 0 : (ox > (int)cw - 1 ? (int)cw - 1 : ox));
    uint32_t y1 = (uint32_t)(oy < 0 ? 0 : (oy > (int)ch - 1 ? (int)ch - 1 : oy));
    float4 A = c[(size_t)my * cw + mx], B = c[(size_t)my * cw + x1];
    float4 E = c[(size_t)y1 * cw + mx], G = c[(size_t)y1 * cw + x1];
    float r0x = A.x * 0.75f + B.x * 0.25f, r0y = A.y * 0.75f + B.y * 0.25f, r0z = A.z * 0.75f + B.z * 0.25f;
    float r1x = E.x * 0.75f + G.x * 0.25f, r1y = E.y * 0.75f + G.y * 0.25f, r1z = E.z * 0.75f + G.z * 0.25f;
    return make_float4(r0x * 0.75f + r1x * 0.25f, r0y * 0.75f + r1y * 0.25f, r0z * 0.75f + r1z * 0.25f, 0.0f);
}

__global__ void k_bloom_up_batch(float4* hdr, const ObsDev* obs, const uint32_t* pre, uint32_t n, int k) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= __ldg(pre + n)) return;
    uint32_t o = find_obs(pre, n, i);
    const ObsDev& od = obs[o];
    uint32_t l = i - __ldg(pre + o);
    uint32_t w = od.lw[k], x = l % w, y = l / w;
    float4 up = upsample_b(hdr + od.pyr_base + od.loff[k + 1], od.lw[k + 1], od.lh[k + 1], x, y);
    float4* dst = hdr + od.pyr_base + od.loff[k] + l;
    float4 v = *dst;
    *dst = make_float4(v.x + up.x, v.y + up.y, v.z + up.z, 0.0f);
}

// The composite (bloom.rs:93-125) and pack_rgb_with_lut (renderer.rs:1116-1129) of every pixel of
// the batch. A block takes a contiguous run of 256-pixel segments, so a thread's pixels increase
// and it keeps its observer's pyramid fields in registers, looking them up again only when it
// crosses into the next observer; per pixel only the independent HDR loads remain. The block
// stages the gamma LUT in shared memory once (the grid is a few blocks per SM).
__global__ void __launch_bounds__(256) k_bloom_composite_batch(const float4* __restrict__ hdr,
                                                               const ObsDev* __restrict__ obs,
                                                               const uint32_t* __restrict__ pre, uint32_t n,
                                                               uint32_t* __restrict__ rgb, const uint32_t* tables) {
    __shared__ uint8_t lut[SR_GAMMA_LUT_SIZE];
    for (uint32_t i = threadIdx.x; i < SR_GAMMA_LUT_SIZE; i += blockDim.x) lut[i] = (uint8_t)__ldg(tables + i);
    __syncthreads();
    const uint32_t total = __ldg(pre + n);
    const uint32_t segs = (total + blockDim.x - 1) / blockDim.x;
    const uint32_t per = (segs + gridDim.x - 1) / gridDim.x;
    const uint32_t s0 = blockIdx.x * per, s1 = min(segs, s0 + per);
    uint32_t lo = 0, hi = 0, w = 1, w1 = 1, h1 = 1;
    const float4* base0 = hdr;
    const float4* base1 = hdr;
    const float strength = 0.04f;
    const float keep = 1.0f - strength;
    const float halo = strength / (float)SR_BLOOM_LEVELS;
    const float scale = (float)(SR_GAMMA_LUT_SIZE - 1);
    for (uint32_t sg = s0; sg < s1; ++sg) {
        const uint32_t i = sg * blockDim.x + threadIdx.x;
        if (i >= total) break;
        if (i >= hi) {  // the next observer of this thread's run
            const uint32_t o = find_obs(pre, n, i);
            const ObsDev& od = obs[o];
            lo = __ldg(pre + o);
            hi = __ldg(pre + o + 1);
            w = od.lw[0];
            w1 = od.lw[1];
            h1 = od.lh[1];
            base0 = hdr + od.pyr_base;
            base1 = hdr + od.pyr_base + od.loff[1];
        }
        const uint32_t l = i - lo, x = l % w, y = l / w;
        const float4 up = upsample_b(base1, w1, h1, x, y);
        const float4 c = base0[l];
        float cx = c.x * keep + up.x * halo, cy = c.y * keep + up.y * halo, cz = c.z * keep + up.z * halo;
        float mx = cx / (1.0f + cx * 0.35f), my = cy / (1.0f + cy * 0.35f), mz = cz / (1.0f + cz * 0.35f);
        mx = mx < 0.0f ? 0.0f : (mx > 1.0f ? 1.0f : mx);
        my = my < 0.0f ? 0.0f : (my > 1.0f ? 1.0f : my);
        mz = mz < 0.0f ? 0.0f : (mz > 1.0f ? 1.0f : mz);
        float fx = mx * scale, fy = my * scale, fz = mz * scale;
        uint32_t ix = fx > 0.0f ? (uint32_t)fx : 0u, iy = fy > 0.0f ? (uint32_t)fy : 0u, iz = fz > 0.0f ? (uint32_t)fz : 0u;
        rgb[i] = ((uint32_t)lut[ix] << 16) | ((uint32_t)lut[iy] << 8) | (uint32_t)lut[iz];
    }
}

}  // namespace srk
