// FP64 host precompute of the KIFMM translation operators.
//
// Restates fmm/trans.cc (surfaces, kernel matrices, pseudo-inverses) and
// compute_fft_trans (fmm/omp_sse_block.cc:432-478, fmm/omp.cc same logic):
//   - sample surfaces: the boundary nodes of an np^3 grid with step 2/(np-1)
//     on [-R,R]^3, x from the outer loop index (trans.cc:35-63);
//     UE (np,1), UC (np+2,3), DE (np,3), DC (np,1) (trans.cc:14-26);
//   - kernel matrices K[j + i*tn] = 1/(4 pi |x_i - y_j|), x = equivalent
//     (source) points, y = check (target) points (omp.cc:289-318);
//   - UC2UE = pinv(K(UE->UC)), DC2DE = pinv(K(DE->DC)) with the cutoff
//     0.1^(np+1) * sigma_max (trans.cc:107-124, 144-173, 209-236);
//     UE2UC[c]: UE shifted by (2c-1), UC scaled by 2 (trans.cc:175-207);
//     DE2DC[c]: DC scaled by 1/2 and shifted by (c-1/2) (trans.cc:238-268);
//   - translation spectra: r2c DFT of 1/(4 pi |2 delta - g|) sampled on the
//     (2np)^3 wrap-around grid g (trans.cc:65-88), for |delta|_inf >= 2.
// The pseudo-inverse uses a one-sided Jacobi (Hestenes) SVD, a published
// method with high relative accuracy, in place of LAPACK DGESVD.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

#include "host.h"

namespace kfmm {

static void sample_grid(int np, double R, std::vector<double>& out) {
  out.clear();
  const double step = 2.0 / (np - 1);
  const double init = -1.0;
  for (int i = 0; i < np; i++)
    for (int j = 0; j < np; j++)
      for (int k = 0; k < np; k++)
        if (i == 0 || i == np - 1 || j == 0 || j == np - 1 || k == 0 || k == np - 1) {
          double x = init + i * step;
          double y = init + j * step;
          double z = init + k * step;
          out.push_back(R * x);
          out.push_back(R * y);
          out.push_back(R * z);
        }
}

void make_surfaces(int np, Surfaces* s) {
  s->np = np;
  sample_grid(np, 1.0, s->ue);
  sample_grid(np + 2, 3.0, s->uc);
  sample_grid(np, 3.0, s->de);
  sample_grid(np, 1.0, s->dc);
  s->P = (int)s->ue.size() / 3;
  s->Q = (int)s->uc.size() / 3;
  s->G = 8 * np * np * np;
  s->F = (np + 1) * 4 * np * np;
}

// K[j + i*tn] = 1/(4 pi |x_i - y_j|): tn x sn column-major (omp.cc:289-318).
static void kernel_matrix(int sn, const double* x, int tn, const double* y, double* mat) {
  for (int i = 0; i < sn; i++)
    for (int j = 0; j < tn; j++) {
      double dx = x[3 * i] - y[3 * j];
      double dy = x[3 * i + 1] - y[3 * j + 1];
      double dz = x[3 * i + 2] - y[3 * j + 2];
      double r2 = dx * dx + dy * dy + dz * dz;
      double r = std::sqrt(r2);
      mat[j + (size_t)i * tn] = (r != 0) ? kOneOver4Pi / r : 0.0;
    }
}

// Pseudo-inverse of the m x n column-major matrix A (m >= n) keeping singular
// values >= eps * sigma_max; result n x m column-major.
static void pinv(const double* A, int m, int n, double eps, double* R) {
  std::vector<double> U(A, A + (size_t)m * n), V((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) V[(size_t)i * n + i] = 1.0;
  const double tol = 1e-15;
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        double* up = &U[(size_t)p * m];
        double* uq = &U[(size_t)q * m];
        double a = 0, b = 0, g = 0;
        for (int i = 0; i < m; ++i) {
          a += up[i] * up[i];
          b += uq[i] * uq[i];
          g += up[i] * uq[i];
        }
        if (g == 0.0) continue;
        double rel = std::fabs(g) / std::sqrt(a * b);
        off = std::max(off, rel);
        if (rel <= tol) continue;
        double zeta = (b - a) / (2.0 * g);
        double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
        double c = 1.0 / std::sqrt(1.0 + t * t), s = c * t;
        for (int i = 0; i < m; ++i) {
          double x = up[i], y = uq[i];
          up[i] = c * x - s * y;
          uq[i] = s * x + c * y;
        }
        double* vp = &V[(size_t)p * n];
        double* vq = &V[(size_t)q * n];
        for (int i = 0; i < n; ++i) {
          double x = vp[i], y = vq[i];
          vp[i] = c * x - s * y;
          vq[i] = s * x + c * y;
        }
      }
    if (off <= tol) break;
  }
  std::vector<double> sig(n);
  std::vector<int> ord(n);
  for (int j = 0; j < n; ++j) {
    double s2 = 0;
    for (int i = 0; i < m; ++i) s2 += U[(size_t)j * m + i] * U[(size_t)j * m + i];
    sig[j] = std::sqrt(s2);
    ord[j] = j;
  }
  std::sort(ord.begin(), ord.end(), [&](int a, int b) { return sig[a] > sig[b]; });
  const double cutoff = eps * sig[ord[0]];
  std::memset(R, 0, sizeof(double) * (size_t)n * m);
  for (int jj = 0; jj < n; ++jj) {
    int j = ord[jj];
    if (!(sig[j] >= cutoff)) break;
    const double inv2 = 1.0 / (sig[j] * sig[j]);  // u_j = U_j / sig, R += v_j u_j^T / sig
    const double* uj = &U[(size_t)j * m];
    const double* vj = &V[(size_t)j * n];
    for (int c = 0; c < m; ++c) {
      const double w = uj[c] * inv2;
      double* rc = R + (size_t)c * n;
      for (int r = 0; r < n; ++r) rc[r] += vj[r] * w;
    }
  }
}

// r2c DFT of an n^3 real grid (C order, last index fastest) to n*n*(n/2+1).
static void r2c3(int n, const double* in, double* out /* interleaved */) {
  const int h = n / 2 + 1;
  std::vector<double> cs(n), sn(n);
  for (int m = 0; m < n; ++m) {
    cs[m] = std::cos(2.0 * M_PI * m / n);
    sn[m] = std::sin(2.0 * M_PI * m / n);
  }
  std::vector<double> re((size_t)n * n * h), im((size_t)n * n * h);
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b)
      for (int k = 0; k < h; ++k) {
        double ar = 0, ai = 0;
        for (int x = 0; x < n; ++x) {
          int m = (k * x) % n;
          ar += in[((size_t)a * n + b) * n + x] * cs[m];
          ai -= in[((size_t)a * n + b) * n + x] * sn[m];
        }
        re[((size_t)a * n + b) * h + k] = ar;
        im[((size_t)a * n + b) * h + k] = ai;
      }
  std::vector<double> tr(n), ti(n);
  auto line = [&](size_t base, size_t stride) {
    for (int k = 0; k < n; ++k) {
      double ar = 0, ai = 0;
      for (int x = 0; x < n; ++x) {
        int m = (k * x) % n;
        double xr = re[base + x * stride], xi = im[base + x * stride];
        ar += xr * cs[m] + xi * sn[m];
        ai += xi * cs[m] - xr * sn[m];
      }
      tr[k] = ar;
      ti[k] = ai;
    }
    for (int k = 0; k < n; ++k) {
      re[base + k * stride] = tr[k];
      im[base + k * stride] = ti[k];
    }
  };
  for (int a = 0; a < n; ++a)
    for (int k = 0; k < h; ++k) line((size_t)a * n * h + k, h);
  for (int b = 0; b < n; ++b)
    for (int k = 0; k < h; ++k) line((size_t)b * h + k, (size_t)n * h);
  for (size_t i = 0; i < re.size(); ++i) {
    out[2 * i] = re[i];
    out[2 * i + 1] = im[i];
  }
}

static void compute_operators(int np, Operators& op) {
  Surfaces S;
  make_surfaces(np, &S);
  const int P = S.P, Q = S.Q, F = S.F, n = 2 * np;
  op.np = np;
  op.P = P;
  op.Q = Q;
  op.F = F;
  const double eps = std::pow(0.1, np + 1);
  std::vector<double> K((size_t)Q * P);
  // UC2UE
  kernel_matrix(P, S.ue.data(), Q, S.uc.data(), K.data());
  op.uc2ue.assign((size_t)P * Q, 0.0);
  pinv(K.data(), Q, P, eps, op.uc2ue.data());
  // UE2UC[c]
  op.ue2uc.assign((size_t)8 * Q * P, 0.0);
  std::vector<double> chk(S.uc.size()), den(S.ue.size());
  for (size_t i = 0; i < S.uc.size(); ++i) chk[i] = 2.0 * S.uc[i];
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int c = 0; c < 2; ++c) {
        int idx[3] = {a, b, c};
        for (int j = 0; j < P; ++j)
          for (int d = 0; d < 3; ++d) den[3 * j + d] = S.ue[3 * j + d] + (2 * idx[d] - 1) * 1.0;
        kernel_matrix(P, den.data(), Q, chk.data(), &op.ue2uc[(size_t)(c + 2 * b + 4 * a) * Q * P]);
      }
  // DC2DE
  std::vector<double> KD((size_t)P * P);
  kernel_matrix(P, S.de.data(), P, S.dc.data(), KD.data());
  op.dc2de.assign((size_t)P * P, 0.0);
  pinv(KD.data(), P, P, eps, op.dc2de.data());
  // DE2DC[c]
  op.de2dc.assign((size_t)8 * P * P, 0.0);
  std::vector<double> chk2(S.dc.size());
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int c = 0; c < 2; ++c) {
        int idx[3] = {a, b, c};
        for (int j = 0; j < P; ++j)
          for (int d = 0; d < 3; ++d)
            chk2[3 * j + d] = 0.5 * S.dc[3 * j + d] + (idx[d] - 0.5) * 1.0;
        kernel_matrix(P, S.de.data(), P, chk2.data(), &op.de2dc[(size_t)(c + 2 * b + 4 * a) * P * P]);
      }
  // translation spectra
  const double step = 2.0 / (np - 1);
  std::vector<double> grid((size_t)3 * n * n * n);
  size_t cnt = 0;
  for (int k = 0; k < n; k++)
    for (int j = 0; j < n; j++)
      for (int i = 0; i < n; i++) {
        int gi = (i < np) ? i : i - n;
        int gj = (j < np) ? j : j - n;
        int gk = (k < np) ? k : k - n;
        grid[cnt++] = 1.0 * gi * step;
        grid[cnt++] = 1.0 * gj * step;
        grid[cnt++] = 1.0 * gk * step;
      }
  op.ue2dc.assign((size_t)343 * 2 * F, 0.0);
  std::vector<double> tt((size_t)n * n * n);
  for (int i3 = -3; i3 <= 3; i3++)
    for (int i2 = -3; i2 <= 3; i2++)
      for (int i1 = -3; i1 <= 3; i1++) {
        if (!(std::abs(i1) > 1 || std::abs(i2) > 1 || std::abs(i3) > 1)) continue;
        int id = (i1 + 3) + (i2 + 3) * 7 + (i3 + 3) * 49;
        double src[3] = {(double)i1 * 2.0 * 1.0, (double)i2 * 2.0 * 1.0, (double)i3 * 2.0 * 1.0};
        kernel_matrix(1, src, n * n * n, grid.data(), tt.data());
        r2c3(n, tt.data(), &op.ue2dc[(size_t)id * 2 * F]);
      }
}

// On-disk operator cache.  With KFMM_OPERATOR_CACHE=<directory> set, the
// operators of an NP are read from <directory>/kifmm_operators_np<NP>.bin when
// that file is valid, else computed and written there (atomically: a
// temporary file renamed into place).  File: magic, format version, NP,
// pseudo-inverse cutoff exponent (np + 1), P, Q, F, the five arrays in
// Operators order, then a 64-bit FNV-1a checksum of everything before it.  A
// file with any other header, size or checksum is ignored and replaced.
namespace {

constexpr uint64_t kOpsMagic = 0x31534f504d4d464bull;  // "KFMMPOS1"
constexpr int kOpsVersion = 1;

uint64_t fnv1a(const void* data, size_t n, uint64_t h = 1469598103934665603ull) {
  const unsigned char* p = (const unsigned char*)data;
  for (size_t i = 0; i < n; ++i) h = (h ^ p[i]) * 1099511628211ull;
  return h;
}

std::vector<std::vector<double>*> op_arrays(Operators& op) {
  return {&op.uc2ue, &op.ue2uc, &op.dc2de, &op.de2dc, &op.ue2dc};
}

std::string cache_path(int np) {
  const char* dir = std::getenv("KFMM_OPERATOR_CACHE");
  if (!dir || !*dir) return std::string();
  return std::string(dir) + "/kifmm_operators_np" + std::to_string(np) + ".bin";
}

bool load_operators(const std::string& path, int np, Operators& op) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  std::vector<unsigned char> buf;
  unsigned char tmp[1 << 16];
  size_t got;
  while ((got = std::fread(tmp, 1, sizeof tmp, f)) > 0) buf.insert(buf.end(), tmp, tmp + got);
  std::fclose(f);
  int64_t head[8];
  if (buf.size() < sizeof head + 8) return false;
  std::memcpy(head, buf.data(), sizeof head);
  Operators want;
  want.np = np;
  want.P = np * np * np - (np - 2) * (np - 2) * (np - 2);
  want.Q = (np + 2) * (np + 2) * (np + 2) - np * np * np;
  want.F = (np + 1) * 4 * np * np;
  const size_t sizes[5] = {(size_t)want.P * want.Q, (size_t)8 * want.Q * want.P,
                           (size_t)want.P * want.P, (size_t)8 * want.P * want.P,
                           (size_t)343 * 2 * want.F};
  size_t total = 0;
  for (size_t z : sizes) total += z;
  if ((uint64_t)head[0] != kOpsMagic || head[1] != kOpsVersion || head[2] != np ||
      head[3] != np + 1 || head[4] != want.P || head[5] != want.Q || head[6] != want.F ||
      head[7] != (int64_t)total || buf.size() != sizeof head + 8 * total + 8)
    return false;
  uint64_t sum;
  std::memcpy(&sum, buf.data() + buf.size() - 8, 8);
  if (fnv1a(buf.data(), buf.size() - 8) != sum) return false;
  const unsigned char* p = buf.data() + sizeof head;
  auto arrays = op_arrays(want);
  for (int k = 0; k < 5; ++k) {
    arrays[k]->resize(sizes[k]);
    std::memcpy(arrays[k]->data(), p, 8 * sizes[k]);
    p += 8 * sizes[k];
  }
  op = std::move(want);
  return true;
}

void store_operators(const std::string& path, Operators& op) {
  std::vector<unsigned char> buf;
  size_t total = 0;
  for (auto* a : op_arrays(op)) total += a->size();
  const int64_t head[8] = {(int64_t)kOpsMagic, kOpsVersion, op.np, op.np + 1,
                           op.P,               op.Q,        op.F,  (int64_t)total};
  buf.insert(buf.end(), (const unsigned char*)head, (const unsigned char*)head + sizeof head);
  for (auto* a : op_arrays(op))
    buf.insert(buf.end(), (const unsigned char*)a->data(),
               (const unsigned char*)(a->data() + a->size()));
  const uint64_t sum = fnv1a(buf.data(), buf.size());
  buf.insert(buf.end(), (const unsigned char*)&sum, (const unsigned char*)&sum + 8);
  const std::string tmp = path + ".tmp" + std::to_string((long long)std::rand());
  FILE* f = std::fopen(tmp.c_str(), "wb");
  if (!f) return;  // the cache is an optimisation: failures leave it alone
  const bool ok = std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
  if (std::fclose(f) == 0 && ok) std::rename(tmp.c_str(), path.c_str());
  else std::remove(tmp.c_str());
}

}  // namespace

const Operators& operators_for(int np) {
  static std::mutex mu;
  static std::map<int, Operators> cache;
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(np);
  if (it != cache.end()) return it->second;
  Operators& op = cache[np];
  const std::string path = cache_path(np);
  if (!path.empty() && load_operators(path, np, op)) return op;
  compute_operators(np, op);
  if (!path.empty()) store_operators(path, op);
  return op;
}

}  // namespace kfmm

using namespace kfmm;

extern "C" kfmm_status kfmm_sizes(int np, int* P, int* Q, int* F) {
  if (np < 3 || np > 8) {
    set_error("kfmm_sizes: NP must be in 3..8");
    return KFMM_ERR_UNSUPPORTED;
  }
  if (P) *P = np * np * np - (np - 2) * (np - 2) * (np - 2);
  if (Q) *Q = (np + 2) * (np + 2) * (np + 2) - np * np * np;
  if (F) *F = (np + 1) * 4 * np * np;
  return KFMM_OK;
}

extern "C" kfmm_status kfmm_operators(int np, double* uc2ue, double* ue2uc, double* dc2de,
                                      double* de2dc, double* ue2dc) {
  if (np < 3 || np > 8) {
    set_error("kfmm_operators: NP must be in 3..8");
    return KFMM_ERR_UNSUPPORTED;
  }
  const Operators& op = operators_for(np);
  if (uc2ue) std::memcpy(uc2ue, op.uc2ue.data(), sizeof(double) * op.uc2ue.size());
  if (ue2uc) std::memcpy(ue2uc, op.ue2uc.data(), sizeof(double) * op.ue2uc.size());
  if (dc2de) std::memcpy(dc2de, op.dc2de.data(), sizeof(double) * op.dc2de.size());
  if (de2dc) std::memcpy(de2dc, op.de2dc.data(), sizeof(double) * op.de2dc.size());
  if (ue2dc) std::memcpy(ue2dc, op.ue2dc.data(), sizeof(double) * op.ue2dc.size());
  return KFMM_OK;
}
