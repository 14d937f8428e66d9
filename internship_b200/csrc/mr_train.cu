// The learned part: training data from the project's own delta tracker and
// hand-written forward / backward / Adam kernels for the radiance-predictor
// network.
//
//  * k_train_points: MeanFreePathSample + GetDesiredCountSample
//    (dataGen.cu:148-216) on the GPU: rays from a sphere of radius 0.5 towards
//    the volume, up to four Woodcock vertices each over the 256^3 mip level 0
//    (the density dataGen's host code samples), with the reference's jitter /
//    view-direction rules; compacted with a global counter.
//  * k_train_labels: GetSample / GetSamples (core/render.cuh:276-315,
//    core/volume.cu:550-626): multiple-scattering radiance at a point along
//    its view direction, FP64 accumulation over the samples of a label.
//  * k_train_frames: the two random frames NNPredict draws
//    (core/render.cuh:355-369,469-523) for the view and light directions.
//  * k_train_fwd_bwd: one thread per training row: the network of
//    core/radiancePredict.cu:370-485 (first albedo channel) forward in fp32
//    with every pre-activation kept in local memory, the loss
//    (X - log(1 + label/srp))^2 on the head output X, and the backward pass;
//    weight gradients are summed over the warp with shuffles and added to a
//    global fp32 gradient with one atomic per warp and weight.
//  * k_adam: Adam with bias correction on the fp32 master weights.
#include <algorithm>
#include <cmath>

#include "mr_internal.h"
#include "mr_net_layout.cuh"
#include "mr_track.cuh"
#include "mr_train.cuh"

namespace mr {

// ---- training points --------------------------------------------------------------

// dataGen's host DeterminateNextVertex (dataGen.cu:148-172): Woodcock free
// flight in which one draw rk per tentative collision sets both the step
// (t -= log(1 - rk) / S_max) and the acceptance test (S / S_max > rk), unlike
// the renderer's DeterminateNextVertex (core/render.cuh:138-172), which draws
// a second number for the test; the correlation shapes where the training
// points fall, so it is kept.
__device__ __forceinline__ bool next_vertex_datagen(const Medium& m, Rng& rng, float alpha, float g, F3 pos, F3 dir,
                                                    float dis, F3& npos, F3& ndir, TrackStats& st) {
  const float smax = m.max_density * alpha;
  float t = 0;
  int loop = 0;
  bool capped = true;
  while (loop++ < 10000) {
    const float rk = rng.next();
    t -= logf(1 - rk) / smax;
    if (t > dis) { npos = f3(0, 0, 0); ndir = f3(0, 0, 0); return false; }
    const float d = fetch_density(m, pos + (dir * t), st);
    if (d * alpha / smax > rk) { capped = false; break; }
    if (d < 0) t -= d;
  }
  if (capped) ++st.caps;
  const float e0 = rng.next(), e1 = rng.next();
  ndir = hg_sample_dir(e0, e1, dir, g);
  npos = (dir * t) + pos;
  return true;
}

// Six draws per vertex (keep, jitter, 3 x jitter point, view), always taken so
// that a ray's stream does not depend on which branches ran. The jitter is a
// uniform point of the ball of radius 1/128 (hash3box, dataGen.cu:115-118).
__global__ void k_train_points(Medium m, float alpha, float g, uint32_t seed, int n_rays, int cap, float* pos,
                               float* dir, unsigned* count, unsigned* caps) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_rays) return;
  TrackStats st{0, 0};
  Rng rng;
  rng.init(seed, (uint32_t)r, 0u, TAG_GEN);
  const float e0 = rng.next(), e1 = rng.next(), e2 = rng.next(), e3 = rng.next();
  const F3 ori = uniform_sphere(e0, e1) * 0.5f;
  const F3 d = normalize(uniform_sphere(e2, e3) + normalize(ori * -1.0f));
  const float dis = ray_box_offset(ori, d);
  if (dis >= 0) {
    F3 sp = ori + d * dis, rd = d;
    for (int i = 0; i < 4; ++i) {
      const float dd = ray_box_distance(sp, rd);
      F3 np, nd;
      if (!next_vertex_datagen(m, rng, alpha, g, sp, rd, dd, np, nd, st)) break;
      const float uk = rng.next(), uj = rng.next(), j0 = rng.next(), j1 = rng.next(), j2 = rng.next(),
                  uv = rng.next();
      const F3 dv = sp - np;
      if (i == 0 || dot(dv, dv) > 1.0f / 64.0f || uk > 0.9f) {
        F3 p = np;
        if (uj > 0.5f) p = p + uniform_sphere(j0, j1) * (cbrtf(j2) * (1.0f / 128.0f));
        const F3 v = uv > 0.25f ? d : rd;
        const unsigned k = atomicAdd(count, 1u);
        if (k < (unsigned)cap) {
          pos[3 * k] = p.x; pos[3 * k + 1] = p.y; pos[3 * k + 2] = p.z;
          dir[3 * k] = v.x; dir[3 * k + 1] = v.y; dir[3 * k + 2] = v.z;
        }
      }
      sp = np;
      rd = nd;
    }
  }
  if (st.caps) atomicAdd(caps, st.caps);
}

// ---- labels -----------------------------------------------------------------------

struct LabelArgs {
  Medium m;
  const float* pos;
  const float* dir;
  int n, spp, chunk, max_bounces;
  F3 L;
  float alpha, g, albedo;
  uint32_t seed;
  double* sum;
  unsigned long long* queue;  // work counter
  unsigned* caps;
  PathScene env;  // only the environment fields: map, size and scale (black without a map)
};

// Work item = (label k, chunk of `chunk` samples), claimed from a global queue
// so that long and short paths balance across the grid. Sample s of label k
// uses the stream (seed; k, s, ., TAG_LABEL).
__global__ void __launch_bounds__(128) k_train_labels(LabelArgs a) {
  const unsigned long long per = (unsigned long long)((a.spp + a.chunk - 1) / a.chunk);
  const unsigned long long total = per * (unsigned long long)a.n;
  TrackStats st{0, 0};
  for (;;) {
    const unsigned long long w = claim_work(a.queue);
    if (w >= total) break;
    const int k = (int)(w / per);
    const int s0 = (int)(w % per) * a.chunk;
    const int s1 = min(a.spp, s0 + a.chunk);
    const F3 p0 = f3(a.pos[3 * k], a.pos[3 * k + 1], a.pos[3 * k + 2]);
    const F3 d0 = f3(a.dir[3 * k], a.dir[3 * k + 1], a.dir[3 * k + 2]);
    double acc = 0.0;
    for (int s = s0; s < s1; ++s) {
      Rng rng;
      rng.init(a.seed, (uint32_t)k, (uint32_t)s, TAG_LABEL);
      const float e0 = rng.next(), e1 = rng.next();
      F3 rd = hg_sample_dir(e0, e1, d0, a.g);
      F3 sp = p0;
      float rate = 1.0f, res = 0.0f;
      for (int b = 0; b < a.max_bounces; ++b) {
        F3 np, nd;
        float dis = ray_box_distance(sp, rd);
        if (!next_vertex(a.m, rng, a.alpha, a.g, sp, rd, dis, np, nd, st)) {
          // escaped: SkyBox(dir) * rate (core/render.cuh:294-296), channel 0
          if (a.env.env_map) res = res + rate * sky(a.env, rd).x;
          break;
        }
        sp = np;
        rate = rate * 1.001f * a.albedo;
        dis = ray_box_distance(sp, a.L);
        const float ph = hg_phase(dot(rd, a.L), a.g);
        res = res + rate * (transmittance(a.m, rng, sp, a.L, dis, a.alpha, st) * ph);
        rd = nd;
      }
      acc += (double)res;
    }
    atomicAdd(a.sum + k, acc);
  }
  if (st.caps) atomicAdd(a.caps, st.caps);
}

// Frames of NNPredict for view direction dir[k] and light L: stream
// (seed; k, 1, ., TAG_MISC).
__global__ void k_train_frames(const float* dir, int n, F3 L, uint32_t seed, float* frame) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  Rng rng;
  rng.init(seed, (uint32_t)k, 1u, TAG_MISC);
  F3 X, Y, Z, LX, ly, lz;
  frame_from(rng, f3(dir[3 * k], dir[3 * k + 1], dir[3 * k + 2]), X, Y, Z);
  frame_from(rng, L, LX, ly, lz);
  float* f = frame + 12 * (size_t)k;
  f[0] = X.x; f[1] = X.y; f[2] = X.z; f[3] = Y.x; f[4] = Y.y; f[5] = Y.z;
  f[6] = Z.x; f[7] = Z.y; f[8] = Z.z; f[9] = LX.x; f[10] = LX.y; f[11] = LX.z;
}

// ---- network forward / backward ----------------------------------------------------

// Trunk blocks in evaluation order: main trunk (radiancePredict.cu:396-421),
// then the light-direction trunk (:424-437). Per block: width S, mode (0 SE +
// ADD3, 1 SERES + ADD3, 2 SERES + REP3), descriptor offset, pool index, SE
// weights and the three branch layers (density, transmittance, phase).
struct TrainArgs {
  const float* w;       // fp32 master weights (blob layout)
  float* grad;          // fp32 gradient accumulator (blob layout)
  const float* desc;    // n x 576, row-major
  const float* aux;     // n x 5 (g, gamma, srp.xyz)
  const float* label;   // n radiance labels
  int n;
  float inv_batch;      // loss weight 1/n
  float* loss;          // summed (X - T)^2 / n
  float* h0;            // TR_TRUNK_FWD: the head input per row (n x 128), written
  const float* dh0;     // TR_TRUNK_BWD: its gradient per row (n x 128), read
};

// Parts of the training step the kernel runs: the whole network (fp32), or
// the two halves around the tensor-core head of the BF16 step (the trunks'
// forward up to the head input, and the trunks' backward from its gradient,
// the forward recomputed).
enum { TR_FULL = 0, TR_TRUNK_FWD = 1, TR_TRUNK_BWD = 2 };

template <int MODE>
__global__ void __launch_bounds__(128) k_train_fwd_bwd(TrainArgs a) {
  const int k0 = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = k0 < a.n;
  const int k = valid ? k0 : a.n - 1;
  const float* __restrict__ W = a.w;
  float* G = a.grad;
  const float* d = a.desc + (size_t)k * 576;
  const float g = a.aux[5 * (size_t)k], gamma = a.aux[5 * (size_t)k + 1], srp = a.aux[5 * (size_t)k + 2];
  const TrainTables& T = c_tt;

  // ---- forward, keeping what the backward pass needs
  float X[12][3][32], YP[12][3][32], Gt[12][3], HP[12][8], TM[12][8];
  float y[3][32];
  float pool[75];
  float YM[3][32], YL[3][8], CMP[3][32], CLP[3][8];
#pragma unroll 1
  for (int b = 0; b < 12; ++b) {
    const int S = T.S[b], mode = T.mode[b], from = T.from[b];
    float mean[3], mx[3];
    for (int br = 0; br < 3; ++br) {
      float s = 0.0f, m = -10000.0f;
      for (int i = 0; i < S; ++i) {
        const float v = d[br * 192 + from + i];
        s += v;
        m = fmaxf(m, v);
      }
      mean[br] = s / (float)S;
      mx[br] = m;
      pool[T.pid[b] + br] = mean[br];
      pool[36 + T.pid[b] + br] = mx[br];
    }
    const float tmp[8] = {mean[0], mean[1], mean[2], mx[0], mx[1], mx[2], g, gamma};
    float h[8];
    for (int i = 0; i < 8; ++i) {
      float s = 0.0f;
      for (int j = 0; j < 8; ++j) s += tmp[j] * __ldg(W + T.se0[b] + j + i * 8);
      TM[b][i] = tmp[i];
      HP[b][i] = s;
      h[i] = relu(s);
    }
    for (int i = 0; i < 3; ++i) {
      float s = 0.0f;
      for (int j = 0; j < 8; ++j) s += h[j] * __ldg(W + T.se1[b] + j + i * 8);
      Gt[b][i] = sigmoid(s);
    }
    for (int br = 0; br < 3; ++br) {
      for (int i = 0; i < S; ++i) {
        const float v = d[br * 192 + from + i] * Gt[b][br];
        X[b][br][i] = mode == 0 ? v : v + y[br][i];
      }
      dense_fwd(W + T.w[b][br], W + T.b[b][br], X[b][br], S, S, YP[b][br]);
      for (int i = 0; i < S; ++i) {
        const float s = d[br * 192 + from + i];
        if (mode == 2) {
          y[br][i] = relu(YP[b][br][i]);
          y[br][S + i] = s;
        } else {
          y[br][i] = relu(YP[b][br][i]) + s;
        }
      }
    }
    if (b == 7) {
      for (int br = 0; br < 3; ++br) {
        for (int i = 0; i < 32; ++i) YM[br][i] = y[br][i];
        dense_fwd(W + T.l81w[br], W + T.l81b[br], YM[br], 32, 32, CMP[br]);
      }
    }
    if (b == 11) {
      for (int br = 0; br < 3; ++br) {
        for (int i = 0; i < 8; ++i) YL[br][i] = y[br][i];
        dense_fwd(W + T.ld41w[br], W + T.ld41b[br], YL[br], 8, 8, CLP[br]);
      }
    }
  }
  pool[72] = g; pool[73] = gamma; pool[74] = srp;
  float FP[16], SW[16], SPP[6], SP[6], X8P[8];
  dense_fwd(W + T.f1, nullptr, pool, 75, 16, FP);
  for (int j = 0; j < 16; ++j) SW[j] = relu(FP[j]);
  dense_fwd(W + T.f2, nullptr, SW, 16, 6, SPP);
  for (int i = 0; i < 6; ++i) SP[i] = sigmoid(SPP[i]);
  const float gg3[3] = {g, gamma, srp};
  dense_fwd(W + T.ggw, W + T.ggb, gg3, 3, 8, X8P);
  float H0[128];
  for (int br = 0; br < 3; ++br)
    for (int i = 0; i < 32; ++i) H0[32 * br + i] = relu(CMP[br][i]) * SP[br];
  for (int br = 0; br < 3; ++br)
    for (int i = 0; i < 8; ++i) H0[96 + 8 * br + i] = relu(CLP[br][i]) * SP[3 + br];
  for (int i = 0; i < 8; ++i) H0[120 + i] = relu(X8P[i]);
  if constexpr (MODE == TR_TRUNK_FWD) {
    if (valid) {
      float4* o = reinterpret_cast<float4*>(a.h0 + (size_t)k * 128);
      for (int i = 0; i < 32; ++i) o[i] = make_float4(H0[4 * i], H0[4 * i + 1], H0[4 * i + 2], H0[4 * i + 3]);
    }
    return;
  }
  float dH0[128];
  if constexpr (MODE == TR_TRUNK_BWD) {
    const float4* gi = reinterpret_cast<const float4*>(a.dh0 + (size_t)k * 128);
    for (int i = 0; i < 32; ++i) {
      const float4 q = valid ? gi[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      dH0[4 * i] = q.x; dH0[4 * i + 1] = q.y; dH0[4 * i + 2] = q.z; dH0[4 * i + 3] = q.w;
    }
  } else {
    float A1P[128], A1[128], A2P[64], A2[64], A3P[32], A3[32];
    dense_fwd(W + T.lc0w, W + T.lc0b, H0, 128, 128, A1P);
    for (int i = 0; i < 128; ++i) A1[i] = relu(A1P[i]);
    dense_fwd(W + T.lc1w, W + T.lc1b, A1, 128, 64, A2P);
    for (int i = 0; i < 64; ++i) A2[i] = relu(A2P[i]);
    dense_fwd(W + T.lc2w, W + T.lc2b, A2, 64, 32, A3P);
    for (int i = 0; i < 32; ++i) A3[i] = relu(A3P[i]);
    float d3[32], dA3[32], d2[64], dA2[64], d1[128], dA1[128];
    tail_fwd_bwd(W, G, T, A3, a.label[k], srp, valid, a.inv_batch, a.loss, d3);
    for (int i = 0; i < 32; ++i) dA3[i] = A3P[i] > 0.0f ? d3[i] : 0.0f;
    for (int i = 0; i < 64; ++i) d2[i] = 0.0f;
    dense_bwd(W + T.lc2w, G + T.lc2w, G + T.lc2b, A2, dA3, d2, 64, 32);
    for (int i = 0; i < 64; ++i) dA2[i] = A2P[i] > 0.0f ? d2[i] : 0.0f;
    for (int i = 0; i < 128; ++i) d1[i] = 0.0f;
    dense_bwd(W + T.lc1w, G + T.lc1w, G + T.lc1b, A1, dA2, d1, 128, 64);
    for (int i = 0; i < 128; ++i) { dA1[i] = A1P[i] > 0.0f ? d1[i] : 0.0f; dH0[i] = 0.0f; }
    dense_bwd(W + T.lc0w, G + T.lc0w, G + T.lc0b, H0, dA1, dH0, 128, 128);
  }
  // head input: gated combs and LGGS
  float dSP[6] = {0, 0, 0, 0, 0, 0};
  float dCM[3][32], dCL[3][8];
  for (int br = 0; br < 3; ++br)
    for (int i = 0; i < 32; ++i) {
      const float dh = dH0[32 * br + i];
      dSP[br] += dh * relu(CMP[br][i]);
      dCM[br][i] = CMP[br][i] > 0.0f ? dh * SP[br] : 0.0f;
    }
  for (int br = 0; br < 3; ++br)
    for (int i = 0; i < 8; ++i) {
      const float dh = dH0[96 + 8 * br + i];
      dSP[3 + br] += dh * relu(CLP[br][i]);
      dCL[br][i] = CLP[br][i] > 0.0f ? dh * SP[3 + br] : 0.0f;
    }
  {
    float dX8[8];
    for (int i = 0; i < 8; ++i) dX8[i] = X8P[i] > 0.0f ? dH0[120 + i] : 0.0f;
    dense_bwd(W + T.ggw, G + T.ggw, G + T.ggb, gg3, dX8, nullptr, 3, 8);
    float dSPP[6], dSW[16], dFP[16];
    for (int i = 0; i < 6; ++i) dSPP[i] = dSP[i] * SP[i] * (1.0f - SP[i]);
    for (int j = 0; j < 16; ++j) dSW[j] = 0.0f;
    dense_bwd(W + T.f2, G + T.f2, nullptr, SW, dSPP, dSW, 16, 6);
    for (int j = 0; j < 16; ++j) dFP[j] = FP[j] > 0.0f ? dSW[j] : 0.0f;
    dense_bwd(W + T.f1, G + T.f1, nullptr, pool, dFP, nullptr, 75, 16);
  }
  // trunks, last block first; dy holds the gradient of the running y
  float dy[3][32];
#pragma unroll 1
  for (int trunk = 0; trunk < 2; ++trunk) {
    const int last = trunk == 0 ? 11 : 7, first = trunk == 0 ? 8 : 0;
    for (int br = 0; br < 3; ++br)
      for (int i = 0; i < 32; ++i) dy[br][i] = 0.0f;
    if (trunk == 0) {
      for (int br = 0; br < 3; ++br) dense_bwd(W + T.ld41w[br], G + T.ld41w[br], G + T.ld41b[br], YL[br], dCL[br], dy[br], 8, 8);
    } else {
      for (int br = 0; br < 3; ++br) dense_bwd(W + T.l81w[br], G + T.l81w[br], G + T.l81b[br], YM[br], dCM[br], dy[br], 32, 32);
    }
#pragma unroll 1
    for (int b = last; b >= first; --b) {
      const int S = T.S[b], mode = T.mode[b], from = T.from[b];
      float dgate[3];
      for (int br = 0; br < 3; ++br) {
        float dp[32], dx[32];
        for (int o = 0; o < S; ++o) { dp[o] = YP[b][br][o] > 0.0f ? dy[br][o] : 0.0f; dx[o] = 0.0f; }
        dense_bwd(W + T.w[b][br], G + T.w[b][br], G + T.b[b][br], X[b][br], dp, dx, S, S);
        float s = 0.0f;
        for (int i = 0; i < S; ++i) s += dx[i] * d[br * 192 + from + i];
        dgate[br] = s;
        for (int i = 0; i < 32; ++i) dy[br][i] = (mode != 0 && i < S) ? dx[i] : 0.0f;
      }
      float dgp[3], h[8], dh[8];
      for (int i = 0; i < 3; ++i) dgp[i] = dgate[i] * Gt[b][i] * (1.0f - Gt[b][i]);
      for (int j = 0; j < 8; ++j) { h[j] = relu(HP[b][j]); dh[j] = 0.0f; }
      dense_bwd(W + T.se1[b], G + T.se1[b], nullptr, h, dgp, dh, 8, 3);
      for (int j = 0; j < 8; ++j) dh[j] = HP[b][j] > 0.0f ? dh[j] : 0.0f;
      dense_bwd(W + T.se0[b], G + T.se0[b], nullptr, TM[b], dh, nullptr, 8, 8);
    }
  }
}

__global__ void k_adam(float* w, float* m, float* v, float* grad, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = grad[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  grad[i] = 0.0f;
}

struct Trainer {
  float* w = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  float* grad = nullptr;
  float* loss = nullptr;
  int step = 0;
  float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  // MR_PREC_BF16: the head on the tensor cores (mr_train_tc.cu) between the
  // trunks' forward and backward halves, which exchange the head input and
  // its gradient per row through h0 / dh0 (cap rows each).
  int precision = MR_PREC_FP32;
  float* h0 = nullptr;
  float* dh0 = nullptr;
  size_t cap = 0;
  uint8_t* img = nullptr;  // BF16 head weights, rebuilt from w every step
  int* err = nullptr;      // set when a bounded wait of the head kernel gives up
};

int launch_head_tc(const float* w, float* grad, uint8_t* img, const float* h0, float* dh0, const float* aux,
                   const float* label, int n, float inv_batch, float* loss, int* err, cudaStream_t s);
size_t head_image_bytes();

}  // namespace mr

using namespace mr;

struct mr_trainer { Trainer t; };

static int check_volume_ready(const mr_volume* h) {
  if (!h) return set_error(MR_ERR_ARG, "NULL volume");
  if (!h->v.data_set || !h->v.mips_valid) return set_error(MR_ERR_STATE, "volume needs mr_volume_set_data and _update");
  return MR_OK;
}

extern "C" int mr_train_points(mr_volume* h, float alpha, float g, uint32_t seed, int32_t n_rays, int32_t cap,
                               float* dev_pos, float* dev_dir, int32_t* host_count, void* stream) {
  clear_error();
  int rc = check_volume_ready(h);
  if (rc) return rc;
  if (!dev_pos || !dev_dir || !host_count) return set_error(MR_ERR_ARG, "mr_train_points: NULL argument");
  if (n_rays < 0 || cap < 0 || !(alpha > 0.0f)) return set_error(MR_ERR_ARG, "mr_train_points: bad n_rays/cap/alpha");
  Volume* v = &h->v;
  cudaStream_t s = (cudaStream_t)stream;
  MR_CUDA(cudaMemsetAsync(v->d_counters, 0, kCounters * sizeof(unsigned long long), s));
  unsigned* cnt = reinterpret_cast<unsigned*>(v->d_counters + 4);
  unsigned* caps = reinterpret_cast<unsigned*>(v->d_counters + 5);
  // dataGen's Woodcock steps read VolumeRender::DensityAtPosition(0, p): the
  // 256^3 level 0 of the mip pyramid, trilinear with a zero border
  // (core/volume.cu:1495-1497, 675-703), under the density grid's majorant.
  if (n_rays > 0)
    k_train_points<<<(n_rays + 127) / 128, 128, 0, s>>>(Medium{v->mips, 256, v->max_density, 1.0f, 0}, alpha, g,
                                                        seed, n_rays, cap, dev_pos, dev_dir, cnt, caps);
  MR_CUDA(cudaGetLastError());
  unsigned c = 0;
  MR_CUDA(cudaMemcpyAsync(&c, cnt, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  MR_CUDA(cudaStreamSynchronize(s));
  *host_count = (int32_t)std::min<unsigned>(c, (unsigned)cap);
  return MR_OK;
}

extern "C" int mr_train_labels(mr_volume* h, const float* dev_pos, const float* dev_dir, int32_t n, mr_float3 light_dir,
                               float alpha, float g, float albedo, int32_t max_bounces, int32_t spp, uint32_t seed,
                               double* dev_sum, void* stream) {
  clear_error();
  int rc = check_volume_ready(h);
  if (rc) return rc;
  if (!dev_pos || !dev_dir || !dev_sum) return set_error(MR_ERR_ARG, "mr_train_labels: NULL argument");
  if (n < 0 || spp <= 0 || max_bounces < 0 || !(alpha > 0.0f))
    return set_error(MR_ERR_ARG, "mr_train_labels: bad n/spp/max_bounces/alpha");
  if (n == 0) return MR_OK;
  Volume* v = &h->v;
  cudaStream_t s = (cudaStream_t)stream;
  MR_CUDA(cudaMemsetAsync(v->d_counters, 0, kCounters * sizeof(unsigned long long), s));
  LabelArgs a;
  a.m = Medium{v->density, v->res, v->max_density, 1.0f};
  a.pos = dev_pos;
  a.dir = dev_dir;
  a.n = n;
  a.spp = spp;
  a.chunk = std::min(spp, 64);
  a.max_bounces = max_bounces;
  a.L = normalize(to_f3(light_dir));
  a.alpha = alpha;
  a.g = g;
  a.albedo = albedo;
  a.seed = seed;
  a.sum = dev_sum;
  a.queue = v->d_counters + 4;
  a.caps = reinterpret_cast<unsigned*>(v->d_counters + 2);
  a.env = PathScene{};
  a.env.env = f3(1.0f, 1.0f, 1.0f);  // the map at unit scale; black without one
  attach_env(a.env, v);
  k_train_labels<<<sm_count() * 16, 128, 0, s>>>(a);
  MR_CUDA(cudaGetLastError());
  return MR_OK;
}

extern "C" int mr_train_frames(const float* dev_dir, int32_t n, mr_float3 light_dir, uint32_t seed, float* dev_frame,
                               void* stream) {
  clear_error();
  if (!dev_dir || !dev_frame) return set_error(MR_ERR_ARG, "mr_train_frames: NULL argument");
  if (n < 0) return set_error(MR_ERR_ARG, "n < 0");
  if (n == 0) return MR_OK;
  k_train_frames<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(dev_dir, n, normalize(to_f3(light_dir)), seed,
                                                                   dev_frame);
  MR_CUDA(cudaGetLastError());
  return MR_OK;
}

extern "C" int mr_trainer_create(const float* host_weights, size_t count, mr_trainer** out) {
  clear_error();
  if (!out || !host_weights) return set_error(MR_ERR_ARG, "mr_trainer_create: NULL argument");
  *out = nullptr;
  if (count != MR_WEIGHT_TOTAL) return set_error(MR_ERR_ARG, "weight blob has %zu floats, expected %d", count, MR_WEIGHT_TOTAL);
  mr_trainer* h = new mr_trainer();
  Trainer& t = h->t;
  const size_t bytes = MR_WEIGHT_TOTAL * sizeof(float);
  cudaError_t e = cudaMalloc(&t.w, bytes);
  if (e == cudaSuccess) e = cudaMalloc(&t.m, bytes);
  if (e == cudaSuccess) e = cudaMalloc(&t.v, bytes);
  if (e == cudaSuccess) e = cudaMalloc(&t.grad, bytes);
  if (e == cudaSuccess) e = cudaMalloc(&t.loss, sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpy(t.w, host_weights, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(t.m, 0, bytes);
  if (e == cudaSuccess) e = cudaMemset(t.v, 0, bytes);
  if (e == cudaSuccess) e = cudaMemset(t.grad, 0, bytes);
  if (e != cudaSuccess) {
    mr_trainer_destroy(h);
    return set_error(MR_ERR_NOMEM, "mr_trainer_create: %s", cudaGetErrorString(e));
  }
  *out = h;
  return MR_OK;
}

extern "C" int mr_trainer_destroy(mr_trainer* h) {
  if (!h) return MR_OK;
  cudaFree(h->t.w);
  cudaFree(h->t.m);
  cudaFree(h->t.v);
  cudaFree(h->t.grad);
  cudaFree(h->t.loss);
  cudaFree(h->t.h0);
  cudaFree(h->t.dh0);
  cudaFree(h->t.img);
  cudaFree(h->t.err);
  delete h;
  return MR_OK;
}

extern "C" int mr_trainer_set_precision(mr_trainer* h, int32_t precision) {
  clear_error();
  if (!h) return set_error(MR_ERR_ARG, "mr_trainer_set_precision: NULL trainer");
  if (precision != MR_PREC_FP32 && precision != MR_PREC_BF16)
    return set_error(MR_ERR_ARG, "training precision must be MR_PREC_FP32 or MR_PREC_BF16 (got %d)", precision);
  Trainer& t = h->t;
  if (precision == MR_PREC_BF16 && !t.img) {
    MR_CUDA(cudaMalloc(&t.img, head_image_bytes()));
    MR_CUDA(cudaMalloc(&t.err, sizeof(int)));
    MR_CUDA(cudaMemset(t.err, 0, sizeof(int)));
  }
  t.precision = precision;
  return MR_OK;
}

// MR_ERR_TIMEOUT (and a reset) when a bounded wait of the BF16 head gave up.
static int head_error(Trainer& t) {
  if (!t.err) return MR_OK;
  int e = 0;
  MR_CUDA(cudaMemcpy(&e, t.err, sizeof(int), cudaMemcpyDeviceToHost));
  if (!e) return MR_OK;
  MR_CUDA(cudaMemset(t.err, 0, sizeof(int)));
  return set_error(MR_ERR_TIMEOUT, "BF16 training head: an mbarrier wait timed out");
}

static int fwd_bwd(Trainer& t, const float* desc, const float* aux, const float* label, int n, cudaStream_t s) {
  MR_CUDA(cudaMemsetAsync(t.loss, 0, sizeof(float), s));
  TrainArgs a;
  a.w = t.w;
  a.grad = t.grad;
  a.desc = desc;
  a.aux = aux;
  a.label = label;
  a.n = n;
  a.inv_batch = 1.0f / (float)n;
  a.loss = t.loss;
  a.h0 = nullptr;
  a.dh0 = nullptr;
  const unsigned grid = (unsigned)((n + 127) / 128);
  if (t.precision != MR_PREC_BF16) {
    k_train_fwd_bwd<TR_FULL><<<grid, 128, 0, s>>>(a);
    MR_CUDA(cudaGetLastError());
    return MR_OK;
  }
  if ((size_t)n > t.cap) {
    cudaFree(t.h0);
    cudaFree(t.dh0);
    t.h0 = t.dh0 = nullptr;
    t.cap = 0;
    MR_CUDA(cudaMalloc(&t.h0, (size_t)n * 128 * sizeof(float)));
    MR_CUDA(cudaMalloc(&t.dh0, (size_t)n * 128 * sizeof(float)));
    t.cap = (size_t)n;
  }
  a.h0 = t.h0;
  a.dh0 = t.dh0;
  k_train_fwd_bwd<TR_TRUNK_FWD><<<grid, 128, 0, s>>>(a);
  MR_CUDA(cudaGetLastError());
  int rc = launch_head_tc(t.w, t.grad, t.img, t.h0, t.dh0, aux, label, n, a.inv_batch, t.loss, t.err, s);
  if (rc) return rc;
  k_train_fwd_bwd<TR_TRUNK_BWD><<<grid, 128, 0, s>>>(a);
  MR_CUDA(cudaGetLastError());
  return MR_OK;
}

extern "C" int mr_trainer_gradient(mr_trainer* h, const float* dev_desc, const float* dev_aux, const float* dev_label,
                                   int32_t n, float* host_grad, float* host_loss, void* stream) {
  clear_error();
  if (!h || !dev_desc || !dev_aux || !dev_label || !host_grad) return set_error(MR_ERR_ARG, "mr_trainer_gradient: NULL argument");
  if (n <= 0) return set_error(MR_ERR_ARG, "n <= 0");
  cudaStream_t s = (cudaStream_t)stream;
  Trainer& t = h->t;
  MR_CUDA(cudaMemsetAsync(t.grad, 0, MR_WEIGHT_TOTAL * sizeof(float), s));
  int rc = fwd_bwd(t, dev_desc, dev_aux, dev_label, n, s);
  if (rc) return rc;
  MR_CUDA(cudaMemcpyAsync(host_grad, t.grad, MR_WEIGHT_TOTAL * sizeof(float), cudaMemcpyDeviceToHost, s));
  float l = 0.0f;
  MR_CUDA(cudaMemcpyAsync(&l, t.loss, sizeof(float), cudaMemcpyDeviceToHost, s));
  MR_CUDA(cudaMemsetAsync(t.grad, 0, MR_WEIGHT_TOTAL * sizeof(float), s));
  MR_CUDA(cudaStreamSynchronize(s));
  if (host_loss) *host_loss = l;
  return head_error(t);
}

extern "C" int mr_trainer_step(mr_trainer* h, const float* dev_desc, const float* dev_aux, const float* dev_label,
                               int32_t n, float lr, float* host_loss, void* stream) {
  clear_error();
  if (!h || !dev_desc || !dev_aux || !dev_label) return set_error(MR_ERR_ARG, "mr_trainer_step: NULL argument");
  if (n <= 0 || !(lr > 0.0f)) return set_error(MR_ERR_ARG, "mr_trainer_step: bad n / lr");
  cudaStream_t s = (cudaStream_t)stream;
  Trainer& t = h->t;
  int rc = fwd_bwd(t, dev_desc, dev_aux, dev_label, n, s);
  if (rc) return rc;
  ++t.step;
  const float c1 = 1.0f - std::pow(t.b1, (float)t.step), c2 = 1.0f - std::pow(t.b2, (float)t.step);
  k_adam<<<(MR_WEIGHT_TOTAL + 255) / 256, 256, 0, s>>>(t.w, t.m, t.v, t.grad, MR_WEIGHT_TOTAL, lr, t.b1, t.b2, t.eps,
                                                        c1, c2);
  MR_CUDA(cudaGetLastError());
  if (host_loss) {
    float l = 0.0f;
    MR_CUDA(cudaMemcpyAsync(&l, t.loss, sizeof(float), cudaMemcpyDeviceToHost, s));
    MR_CUDA(cudaStreamSynchronize(s));
    *host_loss = l;
    return head_error(t);
  }
  return MR_OK;
}

extern "C" int mr_trainer_weights(const mr_trainer* h, float* host_out, size_t count) {
  clear_error();
  if (!h || !host_out) return set_error(MR_ERR_ARG, "mr_trainer_weights: NULL argument");
  if (count != MR_WEIGHT_TOTAL) return set_error(MR_ERR_ARG, "expected %d floats", MR_WEIGHT_TOTAL);
  MR_CUDA(cudaMemcpy(host_out, h->t.w, MR_WEIGHT_TOTAL * sizeof(float), cudaMemcpyDeviceToHost));
  return MR_OK;
}
