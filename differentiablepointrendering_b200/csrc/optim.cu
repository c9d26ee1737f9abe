// optim.cu -- the optimizer step of Pale's training loop on the device.
//
// python/training.py:685-730 hands the gradients of the adjoint pass to a
// torch optimizer over the seven BVH-ordered parameter arrays with one
// learning rate per group (python/optimizers.py:11-66 and :301-337:
// torch.optim.Adam, torch.optim.SGD with momentum 0.8, or the project's
// MaskedAdam, :70-214), steps it, resets the opacities on a schedule, then
// projects the parameters back onto their constraints
// (verify_parameters_inplane, training.py:326-343: render_hooks.py:32-157
// Gram-Schmidt of the tangent frame with the normal towards +Z, :158-258
// clamps of scale [0.01, 1], albedo and opacity [0, 1], beta [-3, 1]) and
// writes them back without a BVH rebuild (apply_point_optimization).  Here
// one kernel does the update, the reset and the projection per surfel and
// writes the parameters and their asset mirror; the surfel arrays the
// traversal reads are derived from them afterwards.
//
// Arithmetic per component, in float32 as the torch kernels do it (scalars
// that torch keeps in Python floats arrive precomputed in double and
// rounded once):
//   Adam     m += (1-b1) (g - m)                 (lerp_, weight < 0.5)
//            v  = v b2 + ((1-b2) g) g            (mul_, addcmul_)
//            p += -(lr / bc1) (m / (sqrt(v) / sqrt(bc2) + eps))
//   SGD      buf = first ? g : buf mu + g;  p += -lr buf
//   MaskedAdam without masks: Adam with m = m b1 + (1-b1) g.
//   MaskedAdam with the per-surfel mask (any gradient entry nonzero):
//            moments as above only where the mask is set, a step count per
//            surfel t, bc = 1 - b^t in float32, and
//            p -= ((1 / max(bc1, 1e-12)) lr) (m / (sqrt(v) / sqrt(bc2) + eps)).
#include "kernels.h"

namespace pale {

namespace {

inline uint32_t blocks_for(uint64_t n) { return (uint32_t)((n + kBlock - 1) / kBlock); }

// Per-surfel bias terms of the masked Adam branch.
struct Bias {
  float rcp1;   // 1 / max(1 - b1^t, 1e-12)
  float bc2s;   // sqrt(1 - b2^t)
};

__device__ __forceinline__ float step_component(const OptArgs& A, const Bias& b, int group, float p, float g, float* m,
                                                float* v) {
  if (A.mode == kOptSgd) {
    const float buf = A.first ? g : *m * A.momentum + g;
    *m = buf;
    return p + (-A.lr[group]) * buf;
  }
  float mm = *m, vv = *v;
  if (A.mode == kOptAdam) {
    mm = mm + A.one_minus_beta1 * (g - mm);
    vv = vv * A.beta2 + A.one_minus_beta2 * g * g;
  } else if (!A.use_mask) {
    mm = mm * A.beta1 + A.one_minus_beta1 * g;
    vv = vv * A.beta2 + A.one_minus_beta2 * g * g;
  } else {
    mm = mm * A.beta1 + A.one_minus_beta1 * g;
    vv = vv * A.beta2 + A.one_minus_beta2 * (g * g);
    *m = mm;
    *v = vv;
    const float denom = sqrtf(vv) / b.bc2s + A.eps;
    return p - (b.rcp1 * A.lr[group]) * (mm / denom);
  }
  *m = mm;
  *v = vv;
  const float denom = sqrtf(vv) / A.bc2_sqrt + A.eps;
  return p + (-A.step_size[group]) * (mm / denom);
}

__device__ __forceinline__ float sum_sq(const float* g, int w) {
  float s = g[0] * g[0];
  for (int c = 1; c < w; ++c) s = s + g[c] * g[c];
  return s;
}

// torch.clamp: NaN stays NaN.
__device__ __forceinline__ float clamp_keep_nan(float x, float lo, float hi) {
  return x < lo ? lo : (x > hi ? hi : x);
}

__device__ __forceinline__ float norm3(const float* a) { return sqrtf(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }

__global__ void k_optimizer_step(OptArgs A) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const PointsDev& G = A.grads;
  const PointsDev& P = A.params;
  float g[16];
  for (int c = 0; c < 3; ++c) {
    g[c] = G.position[3 * i + c];
    g[3 + c] = G.tangent_u[3 * i + c];
    g[6 + c] = G.tangent_v[3 * i + c];
    g[11 + c] = G.albedo[3 * i + c];
  }
  g[9] = G.scale[2 * i];
  g[10] = G.scale[2 * i + 1];
  g[14] = G.opacity[i];
  g[15] = G.beta[i];

  float pos[3], tu[3], tv[3], sc[2], al[3], op, be;
  for (int c = 0; c < 3; ++c) {
    pos[c] = P.position[3 * i + c];
    tu[c] = P.tangent_u[3 * i + c];
    tv[c] = P.tangent_v[3 * i + c];
    al[c] = P.albedo[3 * i + c];
  }
  sc[0] = P.scale[2 * i];
  sc[1] = P.scale[2 * i + 1];
  op = P.opacity[i];
  be = P.beta[i];

  Bias bias{1.0f, 1.0f};
  bool update = true;
  if (A.mode == kOptMaskedAdam && A.use_mask) {
    // compute_surfel_update_mask (optimizers.py:216-246): the float32 sum of
    // the squared gradient entries, field by field, compared with zero.
    float sq = 0.0f;
    sq = sq + sum_sq(g, 3);
    sq = sq + sum_sq(g + 3, 3);
    sq = sq + sum_sq(g + 6, 3);
    sq = sq + sum_sq(g + 9, 2);
    sq = sq + sum_sq(g + 11, 3);
    sq = sq + g[14] * g[14];
    sq = sq + g[15] * g[15];
    update = sq != 0.0f;
    if (update) {
      const uint32_t t = A.steps[i] + 1;
      A.steps[i] = t;
      const float tf = (float)t;
      const float bc1 = 1.0f - powf(A.beta1, tf);
      const float bc2 = 1.0f - powf(A.beta2, tf);
      bias.rcp1 = 1.0f / fmaxf(bc1, 1e-12f);
      bias.bc2s = sqrtf(bc2);
    }
  }
  if (update) {
    const PointsDev& M = A.m;
    const PointsDev& V = A.v;
    for (int c = 0; c < 3; ++c) {
      const size_t k = 3 * (size_t)i + c;
      pos[c] = step_component(A, bias, 0, pos[c], g[c], M.position + k, V.position + k);
      tu[c] = step_component(A, bias, 1, tu[c], g[3 + c], M.tangent_u + k, V.tangent_u + k);
      tv[c] = step_component(A, bias, 1, tv[c], g[6 + c], M.tangent_v + k, V.tangent_v + k);
      al[c] = step_component(A, bias, 3, al[c], g[11 + c], M.albedo + k, V.albedo + k);
    }
    for (int c = 0; c < 2; ++c) {
      const size_t k = 2 * (size_t)i + c;
      sc[c] = step_component(A, bias, 2, sc[c], g[9 + c], M.scale + k, V.scale + k);
    }
    op = step_component(A, bias, 4, op, g[14], M.opacity + i, V.opacity + i);
    be = step_component(A, bias, 5, be, g[15], M.beta + i, V.beta + i);
  }
  // Opacity reset schedule (training.py:707-711), before the projection.
  if (A.opacity_reset >= 0.0f) op = A.opacity_reset;

  // orthonormalize_tangents_inplace (render_hooks.py:32-157)
  const float nu = fmaxf(norm3(tu), 1e-8f);
  float u[3] = {tu[0] / nu, tu[1] / nu, tu[2] / nu};
  const float proj = tv[0] * u[0] + tv[1] * u[1] + tv[2] * u[2];
  float s[3] = {tv[0] - proj * u[0], tv[1] - proj * u[1], tv[2] - proj * u[2]};
  if (s[0] * s[0] + s[1] * s[1] + s[2] * s[2] < 1e-6f) {
    float a[3] = {0.f, 1.f, 0.f};
    if (!(fabsf(u[1]) < 0.9f)) a[0] = 1.f, a[1] = 0.f;
    const float pa = a[0] * u[0] + a[1] * u[1] + a[2] * u[2];
    for (int c = 0; c < 3; ++c) s[c] = a[c] - pa * u[c];
  }
  const float ns = fmaxf(norm3(s), 1e-8f);
  float w[3] = {s[0] / ns, s[1] / ns, s[2] / ns};
  float nrm[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
  const float nn = fmaxf(norm3(nrm), 1e-8f);
  if ((nrm[0] / nn) * A.ref[0] + (nrm[1] / nn) * A.ref[1] + (nrm[2] / nn) * A.ref[2] < 0.0f)
    for (int c = 0; c < 3; ++c) w[c] = -w[c];
  // verify_scales / albedos / opacities / beta (render_hooks.py:158-258)
  for (int c = 0; c < 2; ++c) sc[c] = clamp_keep_nan(sc[c], 0.01f, 1.0f);
  for (int c = 0; c < 3; ++c) al[c] = clamp_keep_nan(al[c], 0.0f, 1.0f);
  op = clamp_keep_nan(op, 0.0f, 1.0f);
  be = clamp_keep_nan(be, -3.0f, 1.0f);

  const PointsDev& Q = A.asset;
  for (int c = 0; c < 3; ++c) {
    P.position[3 * i + c] = Q.position[3 * i + c] = pos[c];
    P.tangent_u[3 * i + c] = Q.tangent_u[3 * i + c] = u[c];
    P.tangent_v[3 * i + c] = Q.tangent_v[3 * i + c] = w[c];
    P.albedo[3 * i + c] = Q.albedo[3 * i + c] = al[c];
  }
  P.scale[2 * i] = Q.scale[2 * i] = sc[0];
  P.scale[2 * i + 1] = Q.scale[2 * i + 1] = sc[1];
  P.opacity[i] = Q.opacity[i] = op;
  P.beta[i] = Q.beta[i] = be;
  Q.shape[i] = P.shape[i];
}

}  // namespace

void optimizer_step(const OptArgs& a, cudaStream_t s) {
  if (a.n == 0) return;
  k_optimizer_step<<<blocks_for(a.n), kBlock, 0, s>>>(a); note_launch();
}

}  // namespace pale
