// The surrogate MLP on the device: parameters, FP32 training (forward, backward, Adam) with the
// kernels of mlp_train.cuh, and the C-ABI tng_mlp_* entry points.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "mlp.h"
#include "mlp_train.cuh"
#include "tiger_chem.h"
#include "tng_runtime.h"

namespace tng {

static int pad16(int x) { return (x + 15) & ~15; }

int mlp_init(Mlp* m, int device, cudaStream_t stream, int n_in, int n_out, int hidden, int layers, uint64_t seed) {
  m->device = device;
  m->stream = stream;
  m->n_in = n_in;
  m->n_out = n_out;
  m->in_pad = pad16(n_in);
  m->out_pad = pad16(n_out);
  m->hidden = hidden;
  m->nlin = layers + 1;
  int64_t off = 0;
  for (int l = 0; l < m->nlin; ++l) {
    const int fi = l == 0 ? m->in_pad : hidden;
    const int fo = l == m->nlin - 1 ? m->out_pad : hidden;
    m->fan_in[l] = fi;
    m->fan_out[l] = fo;
    m->w_off[l] = off;
    off += (int64_t)fi * fo;
    m->b_off[l] = off;
    off += fo;
  }
  m->nparam = off;
  // PyTorch-Linear-style uniform init on the true fan-in, zeros on the padding
  std::vector<float> h(m->nparam, 0.f);
  std::mt19937_64 rng(seed);
  for (int l = 0; l < m->nlin; ++l) {
    const int fi = m->fan_in[l], fo = m->fan_out[l];
    const int fi_true = l == 0 ? n_in : hidden;
    const int fo_true = l == m->nlin - 1 ? n_out : hidden;
    const float bound = 1.0f / std::sqrt((float)fi_true);
    std::uniform_real_distribution<float> U(-bound, bound);
    for (int o = 0; o < fo_true; ++o) {
      for (int i = 0; i < fi_true; ++i) h[m->w_off[l] + (int64_t)o * fi + i] = U(rng);
      h[m->b_off[l] + o] = U(rng);
    }
  }
  cudaError_t e;
  if ((e = cudaMalloc(&m->params, sizeof(float) * m->nparam * 4)) != cudaSuccess) return cuda_error(e, "mlp params");
  m->grads = m->params + m->nparam;
  m->adam_m = m->grads + m->nparam;
  m->adam_v = m->adam_m + m->nparam;
  cudaMemcpy(m->params, h.data(), sizeof(float) * m->nparam, cudaMemcpyHostToDevice);
  cudaMemset(m->grads, 0, sizeof(float) * m->nparam * 3);
  m->step = 0;
  return TNG_OK;
}

void mlp_free(Mlp* m) {
  if (m->params) cudaFree(m->params);
  m->params = nullptr;
  for (DevBuf* b : {&m->act, &m->pre, &m->work, &m->part, &m->lossp, &m->gather}) b->release();
}

static int ensure_work(Mlp* m, int rows) {
  const int H = m->hidden;
  const size_t act = (size_t)rows * (m->in_pad + (size_t)(m->nlin - 1) * H + m->out_pad);
  const size_t pre = (size_t)rows * (m->nlin - 1) * H;
  const size_t work = (size_t)rows * (3 * (size_t)std::max(H, m->out_pad));
  const size_t part = (size_t)32 * H * std::max(H, m->in_pad);
  bool ok = m->act.reserve(act * sizeof(float)) && m->pre.reserve(pre * sizeof(float)) &&
            m->work.reserve(work * sizeof(float)) && m->part.reserve(part * sizeof(float)) &&
            m->lossp.reserve(1024 * sizeof(float));
  if (!ok) return set_error(TNG_ERR_CUDA, "mlp work buffers for %d rows", rows);
  return TNG_OK;
}

static dim3 gemm_grid(int M, int N, int nz = 1) { return dim3((N + kBN - 1) / kBN, (M + kBM - 1) / kBM, nz); }

// activations: H0 (rows x in_pad), H1..H_{nlin-1} (rows x hidden), Y (rows x out_pad)
static float* act_ptr(Mlp* m, int rows, int l) {
  float* a = (float*)m->act.ptr;
  if (l == 0) return a;
  a += (size_t)rows * m->in_pad;
  if (l < m->nlin) return a + (size_t)(l - 1) * rows * m->hidden;
  return a + (size_t)(m->nlin - 1) * rows * m->hidden;
}

static float* pre_ptr(Mlp* m, int rows, int l) { return (float*)m->pre.ptr + (size_t)l * rows * m->hidden; }

int mlp_forward_f32(Mlp* m, const float* X, int rows, float** Yout) {
  int rc = ensure_work(m, rows);
  if (rc) return rc;
  cudaStream_t st = m->stream;
  cudaMemcpyAsync(act_ptr(m, rows, 0), X, sizeof(float) * rows * m->in_pad, cudaMemcpyDeviceToDevice, st);
  for (int l = 0; l < m->nlin; ++l) {
    const int fi = m->fan_in[l], fo = m->fan_out[l];
    const float* W = m->params + m->w_off[l];
    const float* b = m->params + m->b_off[l];
    float* Hin = act_ptr(m, rows, l);
    float* Hout = act_ptr(m, rows, l + 1);
    if (l < m->nlin - 1)
      k_sgemm<0, 1, 2><<<gemm_grid(rows, fo), 256, 0, st>>>(rows, fo, fi, Hin, fi, W, fi, Hout, fo, b,
                                                            pre_ptr(m, rows, l), fi);
    else
      k_sgemm<0, 1, 1><<<gemm_grid(rows, fo), 256, 0, st>>>(rows, fo, fi, Hin, fi, W, fi, Hout, fo, b, nullptr, fi);
  }
  *Yout = act_ptr(m, rows, m->nlin);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TNG_OK : cuda_error(e, "mlp forward");
}

// forward + backward into m->grads; loss (mean weighted squared error) to *loss (host, synchronises)
int mlp_backward(Mlp* m, const float* X, const float* T, const float* w_out, int rows, float* loss) {
  float* Y;
  int rc = mlp_forward_f32(m, X, rows, &Y);
  if (rc) return rc;
  cudaStream_t st = m->stream;
  const int H = m->hidden;
  float* dY = (float*)m->work.ptr;
  float* dA = dY + (size_t)rows * std::max(H, m->out_pad);
  float* dZ = dA + (size_t)rows * std::max(H, m->out_pad);
  const int nb = std::min(1024, (rows * m->out_pad + 255) / 256);
  k_mse<<<nb, 256, 0, st>>>(Y, T, w_out, rows, m->n_out, m->out_pad, m->under_weight, dY, (float*)m->lossp.ptr);
  float* gcur = dY;  // gradient w.r.t. the output of the current layer (pre-activation for the last)
  for (int l = m->nlin - 1; l >= 0; --l) {
    const int fi = m->fan_in[l], fo = m->fan_out[l];
    if (l < m->nlin - 1) {
      const int64_t n = (int64_t)rows * fo;
      k_gelu_back<<<(int)std::min<int64_t>(2048, (n + 255) / 256), 256, 0, st>>>(gcur, pre_ptr(m, rows, l), dZ, n);
      gcur = dZ;
    }
    const float* Hin = act_ptr(m, rows, l);
    // dW (fo x fi) = gcur^T (fo x rows) * Hin (rows x fi), split over rows
    const int nz = std::max(1, std::min(32, rows / 256));
    const int kchunk = (rows + nz - 1) / nz;
    float* part = (float*)m->part.ptr;
    k_sgemm<1, 0, 0><<<gemm_grid(fo, fi, nz), 256, 0, st>>>(fo, fi, rows, gcur, fo, Hin, fi, part, fi, nullptr,
                                                             nullptr, kchunk);
    const int64_t nw = (int64_t)fo * fi;
    k_sum_parts<<<(int)std::min<int64_t>(1024, (nw + 255) / 256), 256, 0, st>>>(part, nz, nw, m->grads + m->w_off[l]);
    k_colsum<<<(fo + 127) / 128, 128, 0, st>>>(gcur, rows, fo, fo, m->grads + m->b_off[l]);
    if (l > 0) {
      // dH (rows x fi) = gcur (rows x fo) * W (fo x fi)
      float* dst = (gcur == dA) ? dY : dA;
      k_sgemm<0, 0, 0><<<gemm_grid(rows, fi), 256, 0, st>>>(rows, fi, fo, gcur, fo, m->params + m->w_off[l], fi,
                                                            dst, fi, nullptr, nullptr, fo);
      gcur = dst;
      if (gcur == dZ) gcur = dA;
    }
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "mlp backward");
  if (loss) {
    std::vector<float> lp(nb);
    cudaMemcpyAsync(lp.data(), m->lossp.ptr, sizeof(float) * nb, cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_error(e, "mlp backward");
    double s = 0.0;
    for (float v : lp) s += v;
    *loss = (float)s;
  }
  return TNG_OK;
}

int mlp_adam(Mlp* m, float lr) {
  m->step += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float bc1 = 1.f - std::pow(b1, (float)m->step), bc2 = 1.f - std::pow(b2, (float)m->step);
  k_adam<<<(int)std::min<int64_t>(2048, (m->nparam + 255) / 256), 256, 0, m->stream>>>(
      m->params, m->grads, m->adam_m, m->adam_v, m->nparam, lr, b1, b2, 1e-8f, bc1, bc2);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TNG_OK : cuda_error(e, "adam");
}

int mlp_train(Mlp* m, const float* X, const float* T, const float* w_out, int64_t n, int epochs, int batch,
              float lr0, uint64_t seed, float* losses, const int* pop, int64_t npop) {
  const int64_t np = pop ? npop : n;
  if (np < batch) batch = (int)np;
  if (batch < 1) return set_error(TNG_ERR_ARG, "mlp train: empty population");
  if (!m->gather.reserve((size_t)batch * (m->in_pad + m->out_pad) * sizeof(float) + sizeof(int) * (size_t)np))
    return set_error(TNG_ERR_CUDA, "mlp gather buffers");
  float* Xb = (float*)m->gather.ptr;
  float* Tb = Xb + (size_t)batch * m->in_pad;
  int* perm_d = (int*)(Tb + (size_t)batch * m->out_pad);
  std::vector<int> perm(np);
  for (int64_t i = 0; i < np; ++i) perm[i] = pop ? pop[i] : (int)i;
  std::mt19937_64 rng(seed);
  const int64_t steps_per_epoch = np / batch;
  const int64_t total = steps_per_epoch * epochs;
  int64_t s = 0;
  for (int ep = 0; ep < epochs; ++ep) {
    std::shuffle(perm.begin(), perm.end(), rng);
    cudaMemcpyAsync(perm_d, perm.data(), sizeof(int) * np, cudaMemcpyHostToDevice, m->stream);
    double lsum = 0.0;
    int nrep = 0;
    for (int64_t b = 0; b < steps_per_epoch; ++b, ++s) {
      const int* idx = perm_d + b * batch;
      k_gather_rows<<<512, 256, 0, m->stream>>>(X, idx, batch, m->in_pad, Xb);
      k_gather_rows<<<512, 256, 0, m->stream>>>(T, idx, batch, m->out_pad, Tb);
      const bool report = (b == steps_per_epoch - 1) || (b % 16 == 0);
      float l = 0.f;
      int rc = mlp_backward(m, Xb, Tb, w_out, batch, report ? &l : nullptr);
      if (rc) return rc;
      // cosine learning-rate schedule
      const float lr = lr0 * 0.5f * (1.f + std::cos(3.14159265358979f * (float)s / (float)std::max<int64_t>(total, 1)));
      if ((rc = mlp_adam(m, lr))) return rc;
      if (report) {
        lsum += l;
        ++nrep;
      }
    }
    if (losses) losses[ep] = (float)(lsum / std::max(nrep, 1));  // mean of the sampled minibatch losses
  }
  cudaError_t e = cudaStreamSynchronize(m->stream);
  return e == cudaSuccess ? TNG_OK : cuda_error(e, "mlp train");
}

}  // namespace tng

using namespace tng;

struct tng_mlp {
  Mlp m;
  tng_chem* h;
};

extern "C" {

int tng_mlp_create(tng_chem* h, int n_in, int n_out, int hidden, int layers, uint64_t seed, tng_mlp** out) {
  if (!h || !out) return set_error(TNG_ERR_ARG, "tng_mlp_create: null argument");
  if (n_in < 1 || n_out < 1 || hidden < 16 || hidden > 256 || hidden % 16 || layers < 1 || layers > kMlpMaxHidden)
    return set_error(TNG_ERR_ARG, "tng_mlp_create: bad sizes");
  DeviceGuard g(h->cfg.device);
  tng_mlp* p = new tng_mlp();
  p->h = h;
  int rc = mlp_init(&p->m, h->cfg.device, h->stream, n_in, n_out, hidden, layers, seed);
  if (rc) {
    delete p;
    return rc;
  }
  h->dependents++;
  *out = p;
  return TNG_OK;
}

int tng_mlp_destroy(tng_mlp* p) {
  if (!p) return TNG_OK;
  DeviceGuard g(p->m.device);
  cudaStreamSynchronize(p->m.stream);
  mlp_free(&p->m);
  p->h->dependents--;
  delete p;
  return TNG_OK;
}

int64_t tng_mlp_param_count(const tng_mlp* p) { return p ? p->m.nparam : 0; }

int tng_mlp_get_params(tng_mlp* p, float* host, int which) {
  if (!p || !host) return set_error(TNG_ERR_ARG, "tng_mlp_get_params: null argument");
  DeviceGuard g(p->m.device);
  const float* src = which == 1 ? p->m.grads : (which == 2 ? p->m.adam_m : (which == 3 ? p->m.adam_v : p->m.params));
  cudaStreamSynchronize(p->m.stream);
  cudaError_t e = cudaMemcpy(host, src, sizeof(float) * p->m.nparam, cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? TNG_OK : cuda_error(e, "tng_mlp_get_params");
}

int tng_mlp_set_params(tng_mlp* p, const float* host) {
  if (!p || !host) return set_error(TNG_ERR_ARG, "tng_mlp_set_params: null argument");
  DeviceGuard g(p->m.device);
  cudaStreamSynchronize(p->m.stream);
  cudaError_t e = cudaMemcpy(p->m.params, host, sizeof(float) * p->m.nparam, cudaMemcpyHostToDevice);
  return e == cudaSuccess ? TNG_OK : cuda_error(e, "tng_mlp_set_params");
}

int tng_mlp_forward(tng_mlp* p, const float* X, int64_t rows, float* Y) {
  if (!p || !X || !Y || rows <= 0 || rows > (1 << 24)) return set_error(TNG_ERR_ARG, "tng_mlp_forward: bad argument");
  DeviceGuard g(p->m.device);
  float* out;
  int rc = mlp_forward_f32(&p->m, X, (int)rows, &out);
  if (rc) return rc;
  cudaMemcpyAsync(Y, out, sizeof(float) * rows * p->m.out_pad, cudaMemcpyDeviceToDevice, p->m.stream);
  return TNG_OK;
}

int tng_mlp_grad(tng_mlp* p, const float* X, const float* T, const float* w_out, int64_t rows, float* loss) {
  if (!p || !X || !T || !w_out || rows <= 0 || rows > (1 << 24)) return set_error(TNG_ERR_ARG, "tng_mlp_grad: bad argument");
  DeviceGuard g(p->m.device);
  return mlp_backward(&p->m, X, T, w_out, (int)rows, loss);
}

int tng_mlp_set_under_weight(tng_mlp* p, float under) {
  if (!p || !(under > 0.f)) return set_error(TNG_ERR_ARG, "tng_mlp_set_under_weight: bad argument");
  p->m.under_weight = under;
  return TNG_OK;
}

int tng_mlp_adam_step(tng_mlp* p, float lr) {
  if (!p) return set_error(TNG_ERR_ARG, "tng_mlp_adam_step: null handle");
  DeviceGuard g(p->m.device);
  return mlp_adam(&p->m, lr);
}

int tng_mlp_train(tng_mlp* p, const float* X, const float* T, const float* w_out, int64_t n, int epochs, int batch,
                  double lr, uint64_t seed, float* losses) {
  if (!p || !X || !T || !w_out || n <= 0 || epochs < 1 || batch < 1 || n > (1LL << 31) - 1)
    return set_error(TNG_ERR_ARG, "tng_mlp_train: bad argument");
  DeviceGuard g(p->m.device);
  return mlp_train(&p->m, X, T, w_out, n, epochs, batch, (float)lr, seed, losses);
}

}  // extern "C"
