// optiBasis force-error functional of ik-SPME with a piecewise cubic Hermite
// interpolation basis, and its gradient with respect to the basis
// coefficients, for a batch of candidate bases, in FP64 on the GPU.
// Reference: IkError.prepare_sum / prepare_sum_deriv / estimate(_deriv)
// (optiBasis/IkError.py:32-136, C++ twin optiBasis/c.src/include/IkError.h),
// HermiteLossFunc(_Bound0) (optiBasis/IkError.py:166-260),
// HermiteBasisHatComput_Norm1(_Bound0) (optiBasis/HatComput.py:155-300),
// symm_hermite (optiBasis/Hermite.py:6-130).
//
//   error(c) = conv sqrt(sum_o1 q2^2 / N)
//   sum_o1   = (2 pi V)^-2 sum_{m != 0, |m_d| <= K_d/2} 2|G(m)|^2 sum_d T_d(m_d)
//   T_d(m)   = sum_{0 < |l| <= l_cut} phi_d(|m + l K_d|)^2 / phi_d(|m|)^2
//   phi_d(k) = hat0_d(k) + sum_b c_b hat_{d,b}(k)       (linear in c)
//
// T_d depends on m_d only, so the triple sum is regrouped as
// sum_d sum_m W_d(m) T_d(m) with W_d(m) the sum of 2|G|^2 over the other two
// mesh indices: W is a K^3 reduction done once per (box, mesh, beta), and one
// evaluation of a candidate is O(K l_cut n_coef).  The hats are the real part
// of the normalised DFT of each basis function sampled on the over-sampled
// grid x_n = n K/M (folded to (-K/2, K/2]), the same samples np.fft sees in
// the reference; here a direct sum over each function's support with exact
// integer reduction of the phase k n mod M.
#include <cmath>
#include <vector>
#include "device_common.cuh"

namespace {

constexpr int IK_THREADS = 256;
constexpr int IK_MAX_COEF = 128;
constexpr size_t IK_SMEM_LIMIT = 160 * 1024;

struct IkBasis {
  double h, CC, delta;  // knot spacing, cut-off, sample spacing K/M
  long long M;          // samples
  int nbin, nk, bound0;
};

__device__ __forceinline__ double h00(double t) { return (1 + 2 * t) * (1 - t) * (1 - t); }
__device__ __forceinline__ double h01(double t) { return t * t * (3.0 - 2.0 * t); }
__device__ __forceinline__ double h10(double t) { return t * (1 - t) * (1 - t); }
__device__ __forceinline__ double h11(double t) { return t * t * (t - 1); }

// value (slope = false) or slope (slope = true) Hermite basis of `knot` at x
__device__ __forceinline__ double hermite(double x, int knot, double h, bool slope) {
  const double s = x / h;
  if (!(s > knot - 1 && s < knot + 1)) return 0.0;
  if (x < knot * h) {
    const double t = s - (double)(knot - 1);
    return slope ? h11(t) * h : h01(t);
  }
  const double t = s - (double)knot;
  return slope ? h10(t) * h : h00(t);
}

// basis function f: 0 = knot 0 value (the constant part), 1..nk value knots,
// nk+1..2nk slope knots; symmetric in x (slopes odd-mirrored)
__device__ double basis_sample(const IkBasis& B, int f, double x) {
  if (f == 0) return hermite(x, 0, B.h, false);
  const bool slope = f > B.nk;
  const int knot = slope ? f - B.nk : f;
  if (knot == B.nbin && (x > B.CC || x < -B.CC)) return 0.0;  // outermost knot cut at |x| = CC
  const double a = hermite(x, knot, B.h, slope), b = hermite(x, -knot, B.h, slope);
  return slope ? a - b : a + b;
}

// hat[f][k] = (1/M) sum_n f(x_n) cos(2 pi k n / M), k = 0..kmax; one block per
// (function, chunk of k); samples of the support staged in shared memory
constexpr int IK_CHUNK = 2048;
__global__ void __launch_bounds__(IK_THREADS)
k_ikerr_hats(IkBasis B, int K, int kmax, long long nlim, double* __restrict__ hat_out /* [1+ncoef][kmax+1] */) {
  __shared__ double fs[IK_CHUNK];
  __shared__ long long ns[IK_CHUNK];
  const int f = blockIdx.x;
  const int k = blockIdx.y * blockDim.x + threadIdx.x;
  const long long M = B.M;
  const double halfK = (double)K / 2.0;
  // samples n = 0..nlim and M-nlim..M-1 (all n when they would overlap)
  const bool all = 2 * nlim + 1 >= M;
  const long long total = all ? M : 2 * nlim + 1;
  double acc = 0.0;
  for (long long c0 = 0; c0 < total; c0 += IK_CHUNK) {
    const int cnt = (int)min((long long)IK_CHUNK, total - c0);
    __syncthreads();
    for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
      const long long q = c0 + t;
      const long long n = all ? q : (q <= nlim ? q : M - (q - nlim));
      double x = (double)n * B.delta;
      if (x > halfK) x -= (double)K;
      fs[t] = basis_sample(B, f, x);
      ns[t] = n;
    }
    __syncthreads();
    if (k <= kmax) {
      for (int t = 0; t < cnt; ++t) {
        const double v = fs[t];
        if (v != 0.0) {
          const long long r = ((long long)k * ns[t]) % M;
          acc += v * cospi(2.0 * (double)r / (double)M);
        }
      }
    }
  }
  if (k <= kmax) hat_out[(size_t)f * (kmax + 1) + k] = acc / (double)M;
}

// W_d(m) = sum over the other two indices of 2 |G(m)|^2 (m != 0),
// |G|^2 = 16 pi^2 |m*|^2 (e^{-pi^2 |m*|^2 / beta^2} / |m*|^2)^2, m* = m_d / L_d
struct IkMesh {
  int K[3];
  double Li[3];
  double beta;
};
__global__ void __launch_bounds__(IK_THREADS)
k_ikerr_weights(IkMesh g, double* W0, double* W1, double* W2) {
  const int d = blockIdx.y;
  const int i = blockIdx.x;
  if (i > g.K[d]) return;  // whole block leaves before any barrier
  const int a = (d + 1) % 3, b = (d + 2) % 3;
  const int na = g.K[a] + 1, nb = g.K[b] + 1;
  int m[3];
  m[d] = i - g.K[d] / 2;
  const double pb2 = M_PI * M_PI / (g.beta * g.beta);
  double acc = 0.0;
  for (int t = threadIdx.x; t < na * nb; t += blockDim.x) {
    m[a] = t / nb - g.K[a] / 2;
    m[b] = t % nb - g.K[b] / 2;
    if (m[0] == 0 && m[1] == 0 && m[2] == 0) continue;
    const double x = m[0] * g.Li[0], y = m[1] * g.Li[1], z = m[2] * g.Li[2];
    const double mm = x * x + y * y + z * z;
    const double expp = exp(-pb2 * mm) / mm;
    acc += 2.0 * (16.0 * M_PI * M_PI * mm * expp * expp);
  }
  __shared__ double sh[IK_THREADS / 32];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sh[w];
    (d == 0 ? W0 : d == 1 ? W1 : W2)[i] = s;
  }
}

struct IkEval {
  const double* hat0[3];  // [kmax+1]
  const double* hats[3];  // [ncoef][kmax+1]
  const double* W[3];     // [K+1]
  int K[3], kmax[3], off[3];
  int l_cut, ncoef;
  double norm;   // 1 / (2 pi V)^2
  double scale;  // conv sqrt(q2^2 / N)
};

__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sh[w];
  return s;  // valid in thread 0
}

// block (c, y): candidate c; y = 0 its value, y = 1 + b its gradient in
// coefficient b.  Every block forms phi_d = hat0_d + c . hats_d in shared
// memory and the value sum over the (axis, m) pairs (a gradient block needs it
// for the square root's derivative); sums are block-reduced in a fixed order.
__global__ void __launch_bounds__(IK_THREADS)
k_ikerr_eval(IkEval e, const double* __restrict__ coeff, double* __restrict__ value,
             double* __restrict__ grad) {
  extern __shared__ double phi[];  // concatenated phi_0, phi_1, phi_2
  __shared__ double sh[IK_THREADS / 32];
  const int c = blockIdx.x;
  if (blockIdx.y > 0 && !grad) return;
  const double* cc = coeff + (size_t)c * e.ncoef;
  for (int d = 0; d < 3; ++d)
    for (int k = threadIdx.x; k <= e.kmax[d]; k += blockDim.x) {
      double v = e.hat0[d][k];
      for (int b = 0; b < e.ncoef; ++b) v += cc[b] * e.hats[d][(size_t)b * (e.kmax[d] + 1) + k];
      phi[e.off[d] + k] = v;
    }
  __syncthreads();
  const int npair = e.K[0] + e.K[1] + e.K[2] + 3;
  auto pair_of = [&](int p, int& d, int& m) {
    d = p <= e.K[0] ? 0 : (p <= e.K[0] + e.K[1] + 1 ? 1 : 2);
    const int i = d == 0 ? p : (d == 1 ? p - e.K[0] - 1 : p - e.K[0] - e.K[1] - 2);
    m = i - e.K[d] / 2;
    return i;
  };
  double acc = 0.0;
  for (int p = threadIdx.x; p < npair; p += blockDim.x) {
    int d, m;
    const int i = pair_of(p, d, m);
    const double* ph = phi + e.off[d];
    const double p0 = ph[abs(m)];
    const double p02i = 1.0 / (p0 * p0);
    double T = 0.0;
    for (int l = -e.l_cut; l <= e.l_cut; ++l) {
      if (l == 0) continue;
      const double pl = ph[abs(m + l * e.K[d])];
      T += pl * pl * p02i;
    }
    acc += e.W[d][i] * T;
  }
  const double s_tot = block_sum(acc, sh);
  __shared__ double s_o1;
  if (threadIdx.x == 0) {
    s_o1 = s_tot * e.norm;
    if (blockIdx.y == 0) value[c] = sqrt(s_o1) * e.scale;
  }
  __syncthreads();
  if (blockIdx.y == 0) return;
  // d T / d c_b = sum_l 2 phi_l B_l / phi_0^2 - 2 phi_l^2 B_0 / phi_0^3
  const double gpref = e.norm * 0.5 / sqrt(s_o1) * e.scale;
  {
    const int b = blockIdx.y - 1;
    double g = 0.0;
    for (int p = threadIdx.x; p < npair; p += blockDim.x) {
      int d, m;
      const int i = pair_of(p, d, m);
      const double* ph = phi + e.off[d];
      const double* hb = e.hats[d] + (size_t)b * (e.kmax[d] + 1);
      const double p0 = ph[abs(m)];
      const double p02i = 1.0 / (p0 * p0), p03i = 1.0 / (p0 * p0 * p0);
      const double b0 = hb[abs(m)];
      double dT = 0.0;
      for (int l = -e.l_cut; l <= e.l_cut; ++l) {
        if (l == 0) continue;
        const int idx = abs(m + l * e.K[d]);
        const double pl = ph[idx];
        dT += 2 * pl * p02i * hb[idx] - 2 * pl * pl * (p03i * b0);
      }
      g += e.W[d][i] * dT;
    }
    const double gs = block_sum(g, sh);
    if (threadIdx.x == 0) grad[(size_t)c * e.ncoef + b] = gs * gpref;
  }
}

}  // namespace

struct md_ikerr {
  int device = 0;
  cudaStream_t stream = nullptr;
  int K[3] = {0, 0, 0}, kmax[3] = {0, 0, 0};
  double L[3] = {0, 0, 0};
  double beta = 0, CC = 0, q2 = 0, natoms = 0;
  int nbin = 0, nk = 0, ncoef = 0, l_cut = 0, bound0 = 0;
  long long over_smpl = 0;
  double* hats[3] = {nullptr, nullptr, nullptr};  // [1 + ncoef][kmax+1]: row 0 = hat0
  double* W[3] = {nullptr, nullptr, nullptr};
  double* d_coeff = nullptr;
  double* d_out = nullptr;  // values [cap] then grads [cap][ncoef]
  int cap = 0;
  size_t smem = 0;
};

static void ikerr_free(md_ikerr* h) {
  for (int d = 0; d < 3; ++d) {
    if (h->hats[d]) cudaFree(h->hats[d]);
    if (h->W[d]) cudaFree(h->W[d]);
  }
  if (h->d_coeff) cudaFree(h->d_coeff);
  if (h->d_out) cudaFree(h->d_out);
  if (h->stream) cudaStreamDestroy(h->stream);
}

extern "C" int md_ikerr_create(md_ikerr** out, const int K[3], const double L[3], double beta, double CC,
                               int nbin, int l_cut, int bound0, int over_smpl, double q2, double natoms,
                               int device) {
  if (!out || !K || !L || !(beta > 0) || !(CC > 0) || nbin < 2 || l_cut < 1 || l_cut > 256 || !(q2 >= 0) ||
      !(natoms > 0)) {
    md_set_error("md_ikerr_create: bad arguments");
    return MD_ERR_BADARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    md_set_error("md_ikerr_create: no CUDA device %d", device);
    return MD_ERR_CUDA;
  }
  MD_CUDA(cudaSetDevice(device));
  md_ikerr* h = new md_ikerr();
  h->device = device;
  h->beta = beta; h->CC = CC; h->q2 = q2; h->natoms = natoms;
  h->nbin = nbin; h->l_cut = l_cut; h->bound0 = bound0 ? 1 : 0;
  h->nk = bound0 ? nbin - 1 : nbin;
  h->ncoef = 2 * h->nk;
  // over-sampling of HermiteLossFunc: int(400 nbin / CC) (optiBasis/IkError.py:185)
  h->over_smpl = over_smpl > 0 ? over_smpl : (long long)(400.0 * ((double)nbin / CC));
  size_t smem = 0;
  for (int d = 0; d < 3; ++d) {
    h->K[d] = K[d];
    h->L[d] = L[d];
    h->kmax[d] = K[d] / 2 + l_cut * K[d];
    smem += sizeof(double) * (h->kmax[d] + 1);
    if (K[d] < 2 || K[d] > 4096 || !(L[d] > 0)) {
      delete h;
      md_set_error("md_ikerr_create: mesh %d or box %g out of range on axis %d", K[d], L[d], d);
      return MD_ERR_BADARG;
    }
    if ((long long)h->kmax[d] >= (long long)K[d] * h->over_smpl) {
      delete h;
      md_set_error("md_ikerr_create: over-sampling %lld too small for l_cut %d (need K/2 + l_cut K < K over_smpl)",
                   h->over_smpl, l_cut);
      return MD_ERR_BADARG;
    }
  }
  if (h->ncoef > IK_MAX_COEF || smem > IK_SMEM_LIMIT) {
    delete h;
    md_set_error("md_ikerr_create: %d coefficients / %zu bytes of hats exceed the supported %d / %zu",
                 2 * (bound0 ? nbin - 1 : nbin), smem, IK_MAX_COEF, IK_SMEM_LIMIT);
    return MD_ERR_BADARG;
  }
  h->smem = smem;
  bool ok = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) == cudaSuccess;
  for (int d = 0; d < 3 && ok; ++d)
    ok = cudaMalloc(&h->hats[d], sizeof(double) * (1 + h->ncoef) * (h->kmax[d] + 1)) == cudaSuccess &&
         cudaMalloc(&h->W[d], sizeof(double) * (K[d] + 1)) == cudaSuccess;
  if (!ok) {
    ikerr_free(h);
    delete h;
    return md_cuda_fail(cudaGetLastError(), "md_ikerr_create allocation");
  }
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(k_ikerr_eval, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  // hats of every basis function along each axis
  for (int d = 0; d < 3; ++d) {
    IkBasis B;
    B.h = CC / nbin;
    B.CC = CC;
    B.M = (long long)K[d] * h->over_smpl;
    B.delta = (double)K[d] / (double)B.M;
    B.nbin = nbin;
    B.nk = h->nk;
    B.bound0 = h->bound0;
    // the widest support is |x| < (nbin + 1) h
    const long long nlim = (long long)ceil((CC + B.h) / B.delta) + 2;
    dim3 grid(1 + h->ncoef, ceil_div(h->kmax[d] + 1, IK_THREADS));
    k_ikerr_hats<<<grid, IK_THREADS, 0, h->stream>>>(B, K[d], h->kmax[d], nlim, h->hats[d]);
  }
  IkMesh g;
  int kmaxall = 0;
  for (int d = 0; d < 3; ++d) {
    g.K[d] = K[d];
    g.Li[d] = 1.0 / L[d];
    kmaxall = K[d] > kmaxall ? K[d] : kmaxall;
  }
  g.beta = beta;
  k_ikerr_weights<<<dim3(kmaxall + 1, 3), IK_THREADS, 0, h->stream>>>(g, h->W[0], h->W[1], h->W[2]);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    ikerr_free(h);
    delete h;
    return md_cuda_fail(e, "md_ikerr_create setup kernels");
  }
  *out = h;
  return MD_OK;
}

extern "C" int md_ikerr_destroy(md_ikerr* h) {
  if (!h) return MD_OK;
  cudaSetDevice(h->device);
  ikerr_free(h);
  delete h;
  return MD_OK;
}

extern "C" int md_ikerr_num_coeffs(md_ikerr* h, int* out) {
  if (!h || !out) return MD_ERR_BADARG;
  *out = h->ncoef;
  return MD_OK;
}

static int ikerr_launch(md_ikerr* h, int C, const double* d_coeff, double* d_val, double* d_grad,
                        cudaStream_t s) {
  IkEval e;
  int off = 0;
  for (int d = 0; d < 3; ++d) {
    e.hat0[d] = h->hats[d];
    e.hats[d] = h->hats[d] + (h->kmax[d] + 1);
    e.W[d] = h->W[d];
    e.K[d] = h->K[d];
    e.kmax[d] = h->kmax[d];
    e.off[d] = off;
    off += h->kmax[d] + 1;
  }
  e.l_cut = h->l_cut;
  e.ncoef = h->ncoef;
  const double V = h->L[0] * h->L[1] * h->L[2];
  e.norm = 1.0 / (2. * M_PI * V * 2. * M_PI * V);
  e.scale = sqrt(h->q2 * h->q2 / h->natoms) * 138.93545756169981341199;
  k_ikerr_eval<<<dim3(C, d_grad ? 1 + h->ncoef : 1), IK_THREADS, h->smem, s>>>(e, d_coeff, d_val, d_grad);
  MD_CHECK_LAUNCH("k_ikerr_eval");
  return MD_OK;
}

extern "C" int md_ikerr_evaluate(md_ikerr* h, int C, const double* coeffs, double* values, double* grads) {
  if (!h || C < 1 || !coeffs || !values) { md_set_error("md_ikerr_evaluate: bad arguments"); return MD_ERR_BADARG; }
  MD_CUDA(cudaSetDevice(h->device));
  if (C > h->cap) {
    if (h->d_coeff) cudaFree(h->d_coeff);
    if (h->d_out) cudaFree(h->d_out);
    h->d_coeff = h->d_out = nullptr;
    h->cap = 0;
    MD_CUDA(cudaMalloc(&h->d_coeff, sizeof(double) * (size_t)C * h->ncoef));
    MD_CUDA(cudaMalloc(&h->d_out, sizeof(double) * (size_t)C * (1 + h->ncoef)));
    h->cap = C;
  }
  double* d_val = h->d_out;
  double* d_grad = grads ? h->d_out + C : nullptr;
  MD_CUDA(cudaMemcpyAsync(h->d_coeff, coeffs, sizeof(double) * (size_t)C * h->ncoef, cudaMemcpyHostToDevice,
                          h->stream));
  if (int r = ikerr_launch(h, C, h->d_coeff, d_val, d_grad, h->stream)) return r;
  MD_CUDA(cudaMemcpyAsync(values, d_val, sizeof(double) * C, cudaMemcpyDeviceToHost, h->stream));
  if (grads)
    MD_CUDA(cudaMemcpyAsync(grads, d_grad, sizeof(double) * (size_t)C * h->ncoef, cudaMemcpyDeviceToHost,
                            h->stream));
  MD_CUDA(cudaStreamSynchronize(h->stream));
  return MD_OK;
}

extern "C" int md_ikerr_evaluate_device(md_ikerr* h, int C, const double* d_coeffs, double* d_values,
                                        double* d_grads, void* stream) {
  if (!h || C < 1 || !d_coeffs || !d_values) {
    md_set_error("md_ikerr_evaluate_device: bad arguments");
    return MD_ERR_BADARG;
  }
  return ikerr_launch(h, C, d_coeffs, d_values, d_grads, stream ? (cudaStream_t)stream : h->stream);
}

extern "C" int md_ikerr_get_hats(md_ikerr* h, int d, double* hat0, double* hats) {
  if (!h || d < 0 || d > 2) return MD_ERR_BADARG;
  MD_CUDA(cudaSetDevice(h->device));
  const size_t n = h->kmax[d] + 1;
  MD_CUDA(cudaStreamSynchronize(h->stream));
  if (hat0) MD_CUDA(cudaMemcpy(hat0, h->hats[d], sizeof(double) * n, cudaMemcpyDeviceToHost));
  if (hats) MD_CUDA(cudaMemcpy(hats, h->hats[d] + n, sizeof(double) * n * h->ncoef, cudaMemcpyDeviceToHost));
  return MD_OK;
}

extern "C" int md_ikerr_get_weights(md_ikerr* h, int d, double* W) {
  if (!h || d < 0 || d > 2 || !W) return MD_ERR_BADARG;
  MD_CUDA(cudaSetDevice(h->device));
  MD_CUDA(cudaStreamSynchronize(h->stream));
  MD_CUDA(cudaMemcpy(W, h->W[d], sizeof(double) * (h->K[d] + 1), cudaMemcpyDeviceToHost));
  return MD_OK;
}
