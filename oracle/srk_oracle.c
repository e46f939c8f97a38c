/*
 * srk_oracle.c — TEST INFRASTRUCTURE ONLY.  FP64 CPU restatement of the
 * reference's algorithms for the resist-shrinkage operator, used as the
 * checker by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg.
 * The product (shrinkage_full_tests_b200) never links or calls this code.
 *
 * Layout: column-major buf[col*H + row] everywhere, kernels K[i*KW + j] with
 * column offset i - KW/2 and row offset j - KW/2 (as in the reference).
 *
 * Followed reference code (file:line in pky8903/shrinkage_full_tests):
 *   conv_valid        adjoint/main_adjoint.cu:70-90      (cpu_conv_valid)
 *   grad_x / grad_y   srk_forward.cuh:429-445            (srk_grad_x/_y)
 *   forward combine   srk_forward.cuh:448-460, adjoint/main_adjoint.cu:321-333
 *   adj_wrt_I         adjoint/srk_adjoint.cuh:25-59      (adjointWrtI_kernel)
 *   adj_wrt_E (true)  adjoint/main_adjoint.cu:206-246    (cpu_adj_wrtE)
 *   adj_wrt_E (fft)   adjoint/srk_adjoint.cuh:169-225,301-382: the stored
 *                     spectrum is applied unconjugated, i.e. a convolution
 *   tangent           tan_tanadj/srk_tangent.cuh:28-52,111-151
 *   tangent-adjoint   tan_tanadj/srk_tangent_adjoint.cuh:4-26,105-159
 *   make_kernel       training/main_cd_training.cu:40-77 (float A&S K1)
 *   precompute freq   srk_forward.cuh:154-203 (pad, fftshift, 2D R2C)
 * Every loop below is written from the formulas those functions implement.
 */
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_MAX_THREADS 256

typedef struct {
  int begin, end;
  void* ctx;
  void (*fn)(void* ctx, int col);
} oracle_slice;

static void* oracle_worker(void* arg) {
  oracle_slice* s = (oracle_slice*)arg;
  for (int c = s->begin; c < s->end; ++c) s->fn(s->ctx, c);
  return NULL;
}

/* Run fn(ctx, c) for c in [0, n) over nthreads threads (contiguous slices). */
static void oracle_parallel(int n, int nthreads, void* ctx, void (*fn)(void*, int)) {
  if (nthreads < 1) nthreads = 1;
  if (nthreads > ORACLE_MAX_THREADS) nthreads = ORACLE_MAX_THREADS;
  if (nthreads > n) nthreads = n > 0 ? n : 1;
  pthread_t th[ORACLE_MAX_THREADS];
  oracle_slice sl[ORACLE_MAX_THREADS];
  for (int t = 0; t < nthreads; ++t) {
    sl[t].begin = (int)((long long)n * t / nthreads);
    sl[t].end = (int)((long long)n * (t + 1) / nthreads);
    sl[t].ctx = ctx;
    sl[t].fn = fn;
  }
  for (int t = 1; t < nthreads; ++t) pthread_create(&th[t], NULL, oracle_worker, &sl[t]);
  oracle_worker(&sl[0]);
  for (int t = 1; t < nthreads; ++t) pthread_join(th[t], NULL);
}

/* ---- central differences (zero outside [0,N)) ---------------------------- */
static double gx_at(const double* I, int N, int c, int r) {
  const double right = (c < N - 1) ? I[(long long)(c + 1) * N + r] : 0.0;
  const double left = (c > 0) ? I[(long long)(c - 1) * N + r] : 0.0;
  return (right - left) * 0.5;
}
static double gy_at(const double* I, int N, int c, int r) {
  const double down = (r < N - 1) ? I[(long long)c * N + r + 1] : 0.0;
  const double up = (r > 0) ? I[(long long)c * N + r - 1] : 0.0;
  return (down - up) * 0.5;
}

void oracle_grad(const double* I, int N, double* Ix, double* Iy) {
  for (int c = 0; c < N; ++c)
    for (int r = 0; r < N; ++r) {
      Ix[(long long)c * N + r] = gx_at(I, N, c, r);
      Iy[(long long)c * N + r] = gy_at(I, N, c, r);
    }
}

/* ---- valid convolution on an output window --------------------------------
 * u[o] = scale * sum_{kx,ky} E[g - k] * G[k + c],  g = o + e,  over the window
 * ox in [ox0, ox0+wx), oy in [oy0, oy0+wy).  Two kernels at once (Gy may be
 * NULL).  out[(ox-ox0)*wy + (oy-oy0)].                                    */
typedef struct {
  const double* E;
  int N;
  const double *Gx, *Gy;
  int KW, e, ox0, oy0, wx, wy;
  double scale;
  double *ux, *uy;
} conv_ctx;

static void conv_col(void* vctx, int i) {
  const conv_ctx* a = (const conv_ctx*)vctx;
  const int c = a->KW / 2, N = a->N, KW = a->KW;
  const int gx = a->ox0 + i + a->e;
  for (int j = 0; j < a->wy; ++j) {
    const int gy = a->oy0 + j + a->e;
    double sx = 0.0, sy = 0.0;
    for (int kx = -c; kx <= c; ++kx) {
      const int x = gx - kx;
      if (x < 0 || x >= N) continue;
      const double* col = a->E + (long long)x * N;
      const double* gxc = a->Gx + (long long)(kx + c) * KW + c;
      const double* gyc = a->Gy ? a->Gy + (long long)(kx + c) * KW + c : NULL;
      for (int ky = -c; ky <= c; ++ky) {
        const int y = gy - ky;
        if (y < 0 || y >= N) continue;
        const double ev = col[y];
        sx += ev * gxc[ky];
        if (gyc) sy += ev * gyc[ky];
      }
    }
    a->ux[(long long)i * a->wy + j] = a->scale * sx;
    if (a->uy) a->uy[(long long)i * a->wy + j] = a->scale * sy;
  }
}

void oracle_conv_window(const double* E, int N, const double* Gx, const double* Gy, int KW, int e, double scale,
                        int ox0, int oy0, int wx, int wy, double* ux, double* uy, int nthreads) {
  conv_ctx a = {E, N, Gx, Gy, KW, e, ox0, oy0, wx, wy, scale, ux, uy};
  oracle_parallel(wx, nthreads, &a, conv_col);
}

/* Forward on a window: R = ux*dI/dx + uy*dI/dy at g = o + e. */
void oracle_forward_window(const double* E, const double* I, int N, const double* Gx, const double* Gy, int KW,
                           int e, double dx, int ox0, int oy0, int wx, int wy, double* R, double* ux_out,
                           double* uy_out, int nthreads) {
  const long long n = (long long)wx * wy;
  double* ux = ux_out ? ux_out : (double*)malloc(sizeof(double) * n);
  double* uy = uy_out ? uy_out : (double*)malloc(sizeof(double) * n);
  oracle_conv_window(E, N, Gx, Gy, KW, e, dx * dx, ox0, oy0, wx, wy, ux, uy, nthreads);
  for (int i = 0; i < wx; ++i)
    for (int j = 0; j < wy; ++j) {
      const int gx = ox0 + i + e, gy = oy0 + j + e;
      const long long o = (long long)i * wy + j;
      R[o] = ux[o] * gx_at(I, N, gx, gy) + uy[o] * gy_at(I, N, gx, gy);
    }
  if (!ux_out) free(ux);
  if (!uy_out) free(uy);
}

/* ---- the reference's own CPU checker form, for timing ----------------------
 * cpu_conv_valid (adjoint/main_adjoint.cu:70-90) is a single-thread float
 * loop: output rows outer, columns inner, kernel rows outer, kernel columns
 * inner, zero outside the image.  This restates it (two kernels, then the
 * combine of :321-333 with the gradient rule) on the output columns
 * [ox0, ox0+wx), so that the measurement can time a bounded sample of an
 * image with the reference's arithmetic type and loop order.  The FP64
 * functions above are the checker.  R[(ox-ox0)*W + oy]. */
static float conv_f32_at(const float* E, int N, const float* G, int KW, int gx, int gy) {
  const int c = KW / 2;
  float sum = 0.f;
  for (int ky = -c; ky <= c; ++ky)
    for (int kx = -c; kx <= c; ++kx) {
      const int y = gy - ky, x = gx - kx;
      if (y >= 0 && y < N && x >= 0 && x < N) sum += E[(long long)x * N + y] * G[(kx + c) * KW + (ky + c)];
    }
  return sum;
}

void oracle_forward_f32_cols(const float* E, const float* I, int N, const float* Gx, const float* Gy, int KW, int e,
                             float dx, int ox0, int wx, float* R) {
  const int W = N - 2 * e;
  const float scale = dx * dx;
  for (int oy = 0; oy < W; ++oy)
    for (int ox = ox0; ox < ox0 + wx; ++ox) {
      const int gx = ox + e, gy = oy + e;
      const float ux = scale * conv_f32_at(E, N, Gx, KW, gx, gy);
      const float uy = scale * conv_f32_at(E, N, Gy, KW, gx, gy);
      const float r = (gx < N - 1) ? I[(long long)(gx + 1) * N + gy] : 0.f;
      const float l = (gx > 0) ? I[(long long)(gx - 1) * N + gy] : 0.f;
      const float d = (gy < N - 1) ? I[(long long)gx * N + gy + 1] : 0.f;
      const float u = (gy > 0) ? I[(long long)gx * N + gy - 1] : 0.f;
      R[(long long)(ox - ox0) * W + oy] = ux * ((r - l) * 0.5f) + uy * ((d - u) * 0.5f);
    }
}

void oracle_forward(const double* E, const double* I, int N, const double* Gx, const double* Gy, int KW, int W,
                    int e, double dx, double* R, double* ux, double* uy, int nthreads) {
  oracle_forward_window(E, I, N, Gx, Gy, KW, e, dx, 0, 0, W, W, R, ux, uy, nthreads);
}

/* ---- adjoint w.r.t. the differentiated field -------------------------------
 * dL/dI[g] = 0.5 (wx[o - ex] - wx[o + ex]) + 0.5 (wy[o - ey] - wy[o + ey]),
 * w = u * v, zero outside the W x W window, o = g - e.                       */
void oracle_adj_wrt_I(const double* wx, const double* wy, int W, int N, int e, double* out) {
#define WAT(arr, r, c) (((r) < 0 || (r) >= W || (c) < 0 || (c) >= W) ? 0.0 : (arr)[(long long)(c) * W + (r)])
  for (int gx = 0; gx < N; ++gx)
    for (int gy = 0; gy < N; ++gy) {
      const int ox = gx - e, oy = gy - e;
      out[(long long)gx * N + gy] = (WAT(wx, oy, ox - 1) - WAT(wx, oy, ox + 1)) * 0.5 +
                                    (WAT(wy, oy - 1, ox) - WAT(wy, oy + 1, ox)) * 0.5;
    }
#undef WAT
}

/* ---- adjoint w.r.t. the convolved field ----------------------------------
 * h_x[g] = v[o] Ix[g] + (dv[o] Ix'[g] ...), only on the valid window.
 * true   : out[p] = dx^2 sum_g (h_x[g] Gx[g - p + c] + h_y[g] Gy[g - p + c])
 * fft    : out[p] = dx^2 sum_g (h_x[g] Gx[p - g + c] + h_y[g] Gy[p - g + c])
 * The caller passes h_x, h_y as full N x N arrays (zero off the window).   */
typedef struct {
  const double *hx, *hy, *Gx, *Gy;
  int N, KW, W, e, fft_conv;
  double scale;
  double* out;
} adjE_ctx;

static void adjE_col(void* vctx, int px) {
  const adjE_ctx* a = (const adjE_ctx*)vctx;
  const int c = a->KW / 2, N = a->N, KW = a->KW, e = a->e, W = a->W;
  for (int py = 0; py < N; ++py) {
    double s = 0.0;
    for (int d = -c; d <= c; ++d) {        /* column offset g - p */
      const int gx = px + d;
      if (gx < e || gx >= e + W) continue;
      const int kx = a->fft_conv ? (-d + c) : (d + c);
      const double* hxc = a->hx + (long long)gx * N;
      const double* hyc = a->hy + (long long)gx * N;
      const double* gxk = a->Gx + (long long)kx * KW;
      const double* gyk = a->Gy + (long long)kx * KW;
      for (int f = -c; f <= c; ++f) {      /* row offset */
        const int gy = py + f;
        if (gy < e || gy >= e + W) continue;
        const int ky = a->fft_conv ? (-f + c) : (f + c);
        s += hxc[gy] * gxk[ky] + hyc[gy] * gyk[ky];
      }
    }
    a->out[(long long)px * N + py] = a->scale * s;
  }
}

void oracle_adj_wrt_E_h(const double* hx, const double* hy, const double* Gx, const double* Gy, int KW, int N,
                        int W, int e, double dx, int fft_conv, double* out, int nthreads) {
  adjE_ctx a = {hx, hy, Gx, Gy, N, KW, W, e, fft_conv, dx * dx, out};
  oracle_parallel(N, nthreads, &a, adjE_col);
}

/* v [W x W], I [N x N] -> dL/dE [N x N] */
void oracle_adj_wrt_E(const double* v, const double* I, const double* Gx, const double* Gy, int KW, int N, int W,
                      int e, double dx, int fft_conv, double* out, int nthreads) {
  const long long nn = (long long)N * N;
  double* hx = (double*)calloc(nn, sizeof(double));
  double* hy = (double*)calloc(nn, sizeof(double));
  for (int ox = 0; ox < W; ++ox)
    for (int oy = 0; oy < W; ++oy) {
      const int gx = ox + e, gy = oy + e;
      const double vv = v[(long long)ox * W + oy];
      hx[(long long)gx * N + gy] = vv * gx_at(I, N, gx, gy);
      hy[(long long)gx * N + gy] = vv * gy_at(I, N, gx, gy);
    }
  oracle_adj_wrt_E_h(hx, hy, Gx, Gy, KW, N, W, e, dx, fft_conv, out, nthreads);
  free(hx);
  free(hy);
}

/* adjointSRK: both outputs, given v, ux, uy (W x W), I (N x N). */
void oracle_adjoint_srk(const double* v, const double* ux, const double* uy, const double* I, const double* Gx,
                        const double* Gy, int KW, int N, int W, int e, double dx, int fft_conv, double* dLdI,
                        double* dLdE, int nthreads) {
  const long long ww = (long long)W * W;
  double* wx = (double*)malloc(sizeof(double) * ww);
  double* wy = (double*)malloc(sizeof(double) * ww);
  for (long long i = 0; i < ww; ++i) { wx[i] = ux[i] * v[i]; wy[i] = uy[i] * v[i]; }
  oracle_adj_wrt_I(wx, wy, W, N, e, dLdI);
  free(wx);
  free(wy);
  oracle_adj_wrt_E(v, I, Gx, Gy, KW, N, W, e, dx, fft_conv, dLdE, nthreads);
}

/* ---- tangent -------------------------------------------------------------- */
void oracle_tangent(const double* f, const double* g, const double* df, const double* dg, const double* Gx,
                    const double* Gy, int KW, int N, int W, int e, double dx, double* dh, int nthreads) {
  const long long ww = (long long)W * W;
  double* buf = (double*)malloc(sizeof(double) * 4 * ww);
  double *uxg = buf, *uyg = buf + ww, *uxd = buf + 2 * ww, *uyd = buf + 3 * ww;
  oracle_conv_window(g, N, Gx, Gy, KW, e, dx * dx, 0, 0, W, W, uxg, uyg, nthreads);
  oracle_conv_window(dg, N, Gx, Gy, KW, e, dx * dx, 0, 0, W, W, uxd, uyd, nthreads);
  for (int ox = 0; ox < W; ++ox)
    for (int oy = 0; oy < W; ++oy) {
      const int gx = ox + e, gy = oy + e;
      const long long o = (long long)ox * W + oy;
      dh[o] = uxd[o] * gx_at(f, N, gx, gy) + uyd[o] * gy_at(f, N, gx, gy) + uxg[o] * gx_at(df, N, gx, gy) +
              uyg[o] * gy_at(df, N, gx, gy);
    }
  free(buf);
}

/* ---- tangent-adjoint -----------------------------------------------------
 * dlam_f = adjWrtI(dlam, ux_g, uy_g) + adjWrtI(lam, ux_dg, uy_dg)
 * dlam_g = adjWrtE(dlam, f) + adjWrtE(lam, df)                             */
void oracle_tangent_adjoint(const double* f, const double* g, const double* df, const double* dg,
                            const double* lam, const double* dlam, const double* Gx, const double* Gy, int KW, int N,
                            int W, int e, double dx, int fft_conv, double* dlf, double* dlg, int nthreads) {
  const long long ww = (long long)W * W, nn = (long long)N * N;
  double* buf = (double*)malloc(sizeof(double) * 6 * ww);
  double *uxg = buf, *uyg = buf + ww, *uxd = buf + 2 * ww, *uyd = buf + 3 * ww, *wx = buf + 4 * ww,
         *wy = buf + 5 * ww;
  oracle_conv_window(g, N, Gx, Gy, KW, e, dx * dx, 0, 0, W, W, uxg, uyg, nthreads);
  oracle_conv_window(dg, N, Gx, Gy, KW, e, dx * dx, 0, 0, W, W, uxd, uyd, nthreads);
  for (long long i = 0; i < ww; ++i) {
    wx[i] = dlam[i] * uxg[i] + lam[i] * uxd[i];
    wy[i] = dlam[i] * uyg[i] + lam[i] * uyd[i];
  }
  oracle_adj_wrt_I(wx, wy, W, N, e, dlf);
  free(buf);
  double* hx = (double*)calloc(nn, sizeof(double));
  double* hy = (double*)calloc(nn, sizeof(double));
  for (int ox = 0; ox < W; ++ox)
    for (int oy = 0; oy < W; ++oy) {
      const int gx = ox + e, gy = oy + e;
      const long long o = (long long)ox * W + oy, q = (long long)gx * N + gy;
      hx[q] = dlam[o] * gx_at(f, N, gx, gy) + lam[o] * gx_at(df, N, gx, gy);
      hy[q] = dlam[o] * gy_at(f, N, gx, gy) + lam[o] * gy_at(df, N, gx, gy);
    }
  oracle_adj_wrt_E_h(hx, hy, Gx, Gy, KW, N, W, e, dx, fft_conv, dlg, nthreads);
  free(hx);
  free(hy);
}

/* ---- kernel generation as the reference does it (float arithmetic) -------
 * Abramowitz & Stegun 9.8.3 (I1, |x|<=3.75), 9.8.7 (K1, x<=2), 9.8.8 (K1,
 * x>2) polynomial coefficients, radial Blackman window, coefficient
 * gamma/(2 pi); zero for r < 1e-6 dx and r > Rw.  Computed in float so the
 * kernel values equal the reference's (training/main_cd_training.cu:40-77). */
static float as_i1_small(float x) {
  const float y = (x / 3.75f) * (x / 3.75f);
  return x * (0.5f + y * (0.87890594f + y * (0.51498869f + y * (0.15084934f +
         y * (0.02658733f + y * (0.00301532f + y * 0.00032411f))))));
}
static float as_k1(float x) {
  if (x <= 0.f) return 1e30f;
  if (x <= 2.f) {
    const float y = x * x * 0.25f, i1 = as_i1_small(x);
    const float p = 1.f + y * (0.15443144f - y * (0.67278579f + y * (0.18156897f +
                    y * (0.01919402f + y * (0.00110404f + y * 0.00004686f)))));
    return logf(x * 0.5f) * i1 + p / x;
  }
  const float y = 2.f / x;
  const float p = 1.25331414f + y * (0.23498619f + y * (-0.03655620f + y * (0.01504268f +
                  y * (-0.00780353f + y * (0.00325614f - y * 0.00068245f)))));
  return expf(-x) / sqrtf(x) * p;
}
static float blackman_f(float r, float Rw) {
  if (r < 0.f || r > Rw) return 0.f;
  const float t = r / Rw;
  return 0.42f + 0.5f * cosf((float)M_PI * t) + 0.08f * cosf(2.f * (float)M_PI * t);
}

/* gamma, Rw in the same length unit as dx; x = (i - kw/2) dx. */
void oracle_make_kernel(int kw, float dx, float gamma, float Rw, float* Kx, float* Ky) {
  const float coeff = gamma / (2.f * (float)M_PI), eps = 1e-6f * dx;
  const int cx = kw / 2;
  memset(Kx, 0, sizeof(float) * kw * kw);
  memset(Ky, 0, sizeof(float) * kw * kw);
  for (int i = 0; i < kw; ++i)
    for (int j = 0; j < kw; ++j) {
      const float x = (i - cx) * dx, y = (j - cx) * dx, r = sqrtf(x * x + y * y);
      if (r < eps || r > Rw) continue;
      const float base = coeff * as_k1(gamma * r) * blackman_f(r, Rw);
      Kx[j + i * kw] = base * (x / r);
      Ky[j + i * kw] = base * (y / r);
    }
}

/* ---- kernel spectrum in the reference layout ------------------------------
 * freq[2*(kx*(M/2+1) + ky) + {0,1}] = sum_{dx,dy} K(dx,dy) e^{-2 pi i (kx dx + ky dy)/M},
 * computed in double (separable two-pass DFT), rounded once to float.      */
void oracle_kernel_freq(const float* K, int kw, int M, float* freq) {
  const int c = kw / 2, H = M / 2 + 1;
  double* cs = (double*)malloc(sizeof(double) * M);
  double* sn = (double*)malloc(sizeof(double) * M);
  for (int m = 0; m < M; ++m) {
    cs[m] = cos(2.0 * M_PI * m / M);
    sn[m] = sin(2.0 * M_PI * m / M);
  }
  /* P[j][kx] = sum_i K[i*kw+j] e^{-2 pi i kx (i-c)/M} */
  double* Pr = (double*)malloc(sizeof(double) * kw * M);
  double* Pi = (double*)malloc(sizeof(double) * kw * M);
  for (int j = 0; j < kw; ++j)
    for (int kx = 0; kx < M; ++kx) {
      double re = 0, im = 0;
      for (int i = 0; i < kw; ++i) {
        const double k = K[i * kw + j];
        if (k == 0.0) continue;
        long long m = ((long long)kx * (i - c)) % M;
        if (m < 0) m += M;
        re += k * cs[m];
        im -= k * sn[m];
      }
      Pr[(long long)j * M + kx] = re;
      Pi[(long long)j * M + kx] = im;
    }
  for (int kx = 0; kx < M; ++kx)
    for (int ky = 0; ky < H; ++ky) {
      double re = 0, im = 0;
      for (int j = 0; j < kw; ++j) {
        long long m = ((long long)ky * (j - c)) % M;
        if (m < 0) m += M;
        const double pr = Pr[(long long)j * M + kx], pi = Pi[(long long)j * M + kx];
        re += pr * cs[m] + pi * sn[m];
        im += pi * cs[m] - pr * sn[m];
      }
      freq[2 * ((long long)kx * H + ky)] = (float)re;
      freq[2 * ((long long)kx * H + ky) + 1] = (float)im;
    }
  free(cs);
  free(sn);
  free(Pr);
  free(Pi);
}
