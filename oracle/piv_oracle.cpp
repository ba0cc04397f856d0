// CPU oracle for the PIV multipass analysis path — TEST INFRASTRUCTURE ONLY (see piv_oracle.h).
//
// Compiled with -ffp-contract=off so that every f32 expression rounds after each operation, as
// the Rust reference does (Rust never contracts a*b+c into an FMA).
//
// The FFT is the one place where the reference's arithmetic lives in a third-party crate that
// is not part of the reference tree: realfft 3.5.0 / rustfft 6.4.1 (rust/Cargo.lock:1644-1646,
// 1703-1705), called at correlate.rs:57-64,152-159,164,173-175. Their published algorithm is an
// unnormalized DFT: X[k] = sum_j x[j] exp(-2 pi i j k / n) forward and the conjugate kernel
// inverse. This file restates that definition with its own mixed-radix recursion; its rounding
// differs from rustfft's, so raw peaks are pinned to a tolerance (1e-4 px), not bit for bit.

#include "piv_oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr uint8_t NO_SIGNAL = 1 << 0;       // field.rs:9
constexpr uint8_t LOW_PPR = 1 << 1;         // field.rs:11
constexpr uint8_t MEDIAN_OUTLIER = 1 << 2;  // field.rs:13
constexpr uint8_t REPLACED = 1 << 3;        // field.rs:15
constexpr uint8_t OUT_OF_RANGE = 1 << 4;    // field.rs:17
constexpr uint8_t INVALID = NO_SIGNAL | LOW_PPR | MEDIAN_OUTLIER | OUT_OF_RANGE;  // field.rs:20
constexpr float MAX_PPR = 1000.0f;          // correlate.rs:24

// Rust's f32::clamp: min if x < min, max if x > max, else x (NaN passes through).
inline float clampf(float x, float lo, float hi) {
    if (x < lo) return lo;
    if (x > hi) return hi;
    return x;
}

// ---------------------------------------------------------------------------------------------
// Grid (grid.rs:20-66)
// ---------------------------------------------------------------------------------------------
inline float center(int64_t origin0, int64_t i, int64_t step, int64_t window) {
    return (float)(origin0 + i * step) + ((float)window - 1.0f) / 2.0f;
}

// ---------------------------------------------------------------------------------------------
// Mixed-radix DFT (definition of the unnormalized DFT; see file header)
// ---------------------------------------------------------------------------------------------
template <class T>
struct FftPlan {
    int n = 0;
    std::vector<int> factors;
    std::vector<std::complex<T>> wf, wi;  // exp(-2 pi i k/n), exp(+2 pi i k/n), twiddles rounded from f64

    explicit FftPlan(int n_) : n(n_) {
        int m = n;
        for (int r : {4, 2, 3, 5}) {
            while (m % r == 0) {
                factors.push_back(r);
                m /= r;
            }
        }
        for (int p = 7; m > 1; p += 2) {
            while (m % p == 0) {
                factors.push_back(p);
                m /= p;
            }
        }
        wf.resize(n);
        wi.resize(n);
        for (int k = 0; k < n; ++k) {
            double a = -2.0 * M_PI * (double)k / (double)n;
            wf[k] = std::complex<T>((T)std::cos(a), (T)std::sin(a));
            wi[k] = std::complex<T>((T)std::cos(a), (T)-std::sin(a));
        }
    }

    // out[k] = sum_j in[j * is] w^(j k), with w = W[stride] (W the n-th roots table of the plan).
    void rec(const std::complex<T>* in, int is, std::complex<T>* out, int len, int fi, int wstep,
             const std::vector<std::complex<T>>& W) const {
        if (len == 1) {
            out[0] = in[0];
            return;
        }
        const int r = factors[fi];
        const int m = len / r;
        for (int q = 0; q < r; ++q) rec(in + q * is, is * r, out + q * m, m, fi + 1, wstep * r, W);
        std::complex<T> t[16];
        std::vector<std::complex<T>> tv;
        std::complex<T>* tp = t;
        if (r > 16) {
            tv.resize(r);
            tp = tv.data();
        }
        for (int k = 0; k < m; ++k) {
            for (int q = 0; q < r; ++q) {
                std::complex<T> v = out[q * m + k];
                if (q != 0 && k != 0) v = cmul(v, W[((int64_t)q * k * wstep) % n]);
                tp[q] = v;
            }
            if (r == 2) {
                out[k] = tp[0] + tp[1];
                out[k + m] = tp[0] - tp[1];
            } else if (r == 4) {
                // w4 = W[n/4 * ...]: forward -i, inverse +i (taken from the table's sign).
                const std::complex<T> j4 = W[(n / 4)];
                std::complex<T> a0 = tp[0] + tp[2], a1 = tp[0] - tp[2];
                std::complex<T> b0 = tp[1] + tp[3], b1 = cmul(tp[1] - tp[3], j4);
                out[k] = a0 + b0;
                out[k + m] = a1 + b1;
                out[k + 2 * m] = a0 - b0;
                out[k + 3 * m] = a1 - b1;
            } else {
                for (int p = 0; p < r; ++p) {
                    std::complex<T> s = tp[0];
                    for (int q = 1; q < r; ++q) s += cmul(tp[q], W[(((int64_t)q * p) % r) * (n / r)]);
                    out[k + p * m] = s;
                }
            }
        }
    }

    static std::complex<T> cmul(std::complex<T> a, std::complex<T> b) {
        return std::complex<T>(a.real() * b.real() - a.imag() * b.imag(),
                               a.real() * b.imag() + a.imag() * b.real());
    }

    // In place via a scratch copy. inverse: conjugate kernel, unnormalized.
    void run(std::complex<T>* x, std::complex<T>* scratch, bool inverse) const {
        std::memcpy(scratch, x, sizeof(std::complex<T>) * n);
        rec(scratch, 1, x, n, 0, 1, inverse ? wi : wf);
    }
};

// ---------------------------------------------------------------------------------------------
// Window load (correlate.rs:182-210)
// ---------------------------------------------------------------------------------------------
double load_window_f32(const float* img, int64_t w, float x, float y, int64_t n, float* dst) {
    const int64_t x0 = (int64_t)std::floor(x), y0 = (int64_t)std::floor(y);
    const float tx = x - (float)x0, ty = y - (float)y0;
    if (tx < 1e-4f && ty < 1e-4f) {
        for (int64_t r = 0; r < n; ++r)
            for (int64_t c = 0; c < n; ++c) dst[r * n + c] = img[(y0 + r) * w + x0 + c];
    } else {
        const float w00 = (1.0f - tx) * (1.0f - ty), w01 = tx * (1.0f - ty), w10 = (1.0f - tx) * ty,
                    w11 = tx * ty;
        for (int64_t r = 0; r < n; ++r) {
            const float* top = img + (y0 + r) * w + x0;
            const float* bot = top + w;
            for (int64_t c = 0; c < n; ++c)
                dst[r * n + c] = w00 * top[c] + w01 * top[c + 1] + w10 * bot[c] + w11 * bot[c + 1];
        }
    }
    double s = 0.0;
    for (int64_t i = 0; i < n * n; ++i) s += (double)dst[i];
    const double mean = s / (double)(n * n);
    double energy = 0.0;
    const float mf = (float)mean;
    for (int64_t i = 0; i < n * n; ++i) {
        dst[i] -= mf;
        energy += (double)dst[i] * (double)dst[i];
    }
    return energy;
}

// FP64 accuracy oracle: the same sampling evaluated in f64.
double load_window_f64(const float* img, int64_t w, float x, float y, int64_t n, double* dst) {
    const int64_t x0 = (int64_t)std::floor(x), y0 = (int64_t)std::floor(y);
    const double tx = (double)x - (double)x0, ty = (double)y - (double)y0;
    if (tx < 1e-4 && ty < 1e-4) {
        for (int64_t r = 0; r < n; ++r)
            for (int64_t c = 0; c < n; ++c) dst[r * n + c] = img[(y0 + r) * w + x0 + c];
    } else {
        const double w00 = (1 - tx) * (1 - ty), w01 = tx * (1 - ty), w10 = (1 - tx) * ty, w11 = tx * ty;
        for (int64_t r = 0; r < n; ++r) {
            const float* top = img + (y0 + r) * w + x0;
            const float* bot = top + w;
            for (int64_t c = 0; c < n; ++c)
                dst[r * n + c] = w00 * top[c] + w01 * top[c + 1] + w10 * bot[c] + w11 * bot[c + 1];
        }
    }
    double s = 0.0;
    for (int64_t i = 0; i < n * n; ++i) s += dst[i];
    const double mean = s / (double)(n * n);
    double energy = 0.0;
    for (int64_t i = 0; i < n * n; ++i) {
        dst[i] -= mean;
        energy += dst[i] * dst[i];
    }
    return energy;
}

// ---------------------------------------------------------------------------------------------
// Peak finding (correlate.rs:215-303), generic over the plane's element type.
// ---------------------------------------------------------------------------------------------
template <class T>
void find_peak_t(const T* corr, int64_t n, T out[4]) {
    auto at = [&](int64_t y, int64_t x) { return corr[(y % n) * n + (x % n)]; };
    auto is_local_max = [&](int64_t y, int64_t x) {
        const T v = at(y, x);
        const int64_t d[8][2] = {{n - 1, n - 1}, {n - 1, 0}, {n - 1, 1}, {0, n - 1},
                                 {0, 1},         {1, n - 1}, {1, 0},     {1, 1}};
        for (auto& e : d)
            if (!(at(y + e[0], x + e[1]) <= v)) return false;
        return true;
    };
    T best = -std::numeric_limits<T>::infinity();
    int64_t by = 0, bx = 0;
    for (int64_t i = 0; i < n * n; ++i) {
        if (corr[i] > best) {
            best = corr[i];
            by = i / n;
            bx = i % n;
        }
    }
    auto half_width = [&](int64_t s0, int64_t s1) {
        int64_t k = 0;
        while (k < n / 2 && at(by + k * s0, bx + k * s1) > (T)0.5 * best) ++k;
        return k;
    };
    int64_t hw = std::max(std::max(half_width(1, 0), half_width(n - 1, 0)),
                          std::max(half_width(0, 1), half_width(0, n - 1)));
    const int64_t exclude = std::max<int64_t>((int64_t)std::ceil(1.5f * (float)hw), 2);
    auto circ = [&](int64_t a, int64_t b) {
        int64_t d = a > b ? a - b : b - a;
        return std::min(d, n - d);
    };
    T second = -std::numeric_limits<T>::infinity();
    for (int64_t y = 0; y < n; ++y)
        for (int64_t x = 0; x < n; ++x) {
            const T v = at(y, x);
            if (v > second && std::max(circ(y, by), circ(x, bx)) > exclude && is_local_max(y, x))
                second = v;
        }
    auto sub = [](T m, T c, T p) -> T {
        T d;
        if (m > 0 && c > 0 && p > 0) {
            const T lm = std::log(m), lc = std::log(c), lp = std::log(p);
            d = (lm - lp) / ((T)2.0 * (lm - (T)2.0 * lc + lp));
        } else {
            d = (m - p) / ((T)2.0 * (m - (T)2.0 * c + p));
        }
        if (std::isfinite(d)) return std::min(std::max(d, (T)-0.5), (T)0.5);
        return (T)0;
    };
    const T sx = sub(at(by, bx + n - 1), best, at(by, bx + 1));
    const T sy = sub(at(by + n - 1, bx), best, at(by + 1, bx));
    auto wrap = [&](int64_t k) { return k >= n / 2 ? (T)k - (T)n : (T)k; };
    const T ppr = second > 0 ? std::min(best / second, (T)MAX_PPR) : (T)MAX_PPR;
    out[0] = wrap(bx) + sx;
    out[1] = wrap(by) + sy;
    out[2] = best;
    out[3] = ppr;
}

// ---------------------------------------------------------------------------------------------
// Correlation (correlate.rs:99-178)
// ---------------------------------------------------------------------------------------------
template <class T>
struct Workspace {
    int64_t n;
    FftPlan<T> plan;
    std::vector<T> a, b, corr;
    std::vector<std::complex<T>> ta, tb, line, scratch;
    std::vector<float> af, bf;
    explicit Workspace(int64_t n_)
        : n(n_), plan((int)n_), a(n_ * n_), b(n_ * n_), corr(n_ * n_), ta((n_ / 2 + 1) * n_),
          tb((n_ / 2 + 1) * n_), line(n_), scratch(n_), af(n_ * n_), bf(n_ * n_) {}

    // forward (correlate.rs:141-160): r2c per row, complex FFT per column; spectra column-major.
    void forward(const T* win, std::vector<std::complex<T>>& out) {
        const int64_t m = n / 2 + 1;
        for (int64_t y = 0; y < n; ++y) {
            for (int64_t x = 0; x < n; ++x) line[x] = std::complex<T>(win[y * n + x], 0);
            plan.run(line.data(), scratch.data(), false);
            for (int64_t c = 0; c < m; ++c) out[c * n + y] = line[c];
        }
        for (int64_t c = 0; c < m; ++c) plan.run(&out[c * n], scratch.data(), false);
    }

    // inverse (correlate.rs:162-178): complex inverse per column, then c2r per row with the
    // DC and Nyquist imaginary parts cleared.
    void inverse() {
        const int64_t m = n / 2 + 1;
        for (int64_t c = 0; c < m; ++c) plan.run(&ta[c * n], scratch.data(), true);
        for (int64_t y = 0; y < n; ++y) {
            for (int64_t c = 0; c < m; ++c) line[c] = ta[c * n + y];
            line[0] = std::complex<T>(line[0].real(), 0);
            line[m - 1] = std::complex<T>(line[m - 1].real(), 0);
            for (int64_t c = m; c < n; ++c) line[c] = std::conj(line[n - c]);
            plan.run(line.data(), scratch.data(), true);
            for (int64_t x = 0; x < n; ++x) corr[y * n + x] = line[x].real();
        }
    }

    // Returns false when either window is flat. Fills corr with the scaled plane.
    bool plane(const float* ia, int64_t wa, float ax, float ay, const float* ib, int64_t wb, float bx,
               float by);
    bool finish(double ea, double eb);
};

template <>
bool Workspace<float>::finish(double ea, double eb);
template <>
bool Workspace<double>::finish(double ea, double eb);

template <>
bool Workspace<float>::plane(const float* ia, int64_t wa, float ax, float ay, const float* ib,
                             int64_t wb, float bx, float by) {
    const double ea = load_window_f32(ia, wa, ax, ay, n, a.data());
    const double eb = load_window_f32(ib, wb, bx, by, n, b.data());
    return finish(ea, eb);
}

// correlate.rs:110-137 on windows already in a and b.
template <>
bool Workspace<float>::finish(double ea, double eb) {
    if (ea <= 1e-12 || eb <= 1e-12) return false;
    forward(a.data(), ta);
    forward(b.data(), tb);
    for (size_t i = 0; i < ta.size(); ++i) ta[i] = FftPlan<float>::cmul(std::conj(ta[i]), tb[i]);
    inverse();
    // correlate.rs:136 — `as` binds tighter than `/`: the f64 denominator is rounded to f32.
    const float scale = 1.0f / (float)((double)(n * n) * std::sqrt(ea * eb));
    for (auto& c : corr) c *= scale;
    return true;
}

template <>
bool Workspace<double>::plane(const float* ia, int64_t wa, float ax, float ay, const float* ib,
                              int64_t wb, float bx, float by) {
    const double ea = load_window_f64(ia, wa, ax, ay, n, a.data());
    const double eb = load_window_f64(ib, wb, bx, by, n, b.data());
    return finish(ea, eb);
}

template <>
bool Workspace<double>::finish(double ea, double eb) {
    if (ea <= 1e-12 || eb <= 1e-12) return false;
    forward(a.data(), ta);
    forward(b.data(), tb);
    for (size_t i = 0; i < ta.size(); ++i) ta[i] = FftPlan<double>::cmul(std::conj(ta[i]), tb[i]);
    inverse();
    const double scale = 1.0 / ((double)(n * n) * std::sqrt(ea * eb));
    for (auto& c : corr) c *= scale;
    return true;
}

// ---------------------------------------------------------------------------------------------
// Integral image (preprocess.rs:76-125), sequential f64 exactly as the reference builds it.
// ---------------------------------------------------------------------------------------------
struct Integral {
    int64_t h, w;
    std::vector<double> sum, sumsq;
    Integral(const float* f, int64_t h_, int64_t w_) : h(h_), w(w_) {
        const int64_t s = w + 1;
        sum.assign(s * (h + 1), 0.0);
        sumsq.assign(s * (h + 1), 0.0);
        for (int64_t y = 0; y < h; ++y) {
            double rs = 0.0, rq = 0.0;
            for (int64_t x = 0; x < w; ++x) {
                const double v = (double)f[y * w + x];
                rs += v;
                rq += v * v;
                const int64_t i = (y + 1) * s + x + 1;
                sum[i] = sum[i - s] + rs;
                sumsq[i] = sumsq[i - s] + rq;
            }
        }
    }
    static double rect(const std::vector<double>& t, int64_t s, int64_t x0, int64_t y0, int64_t x1,
                       int64_t y1) {
        return t[y1 * s + x1] - t[y0 * s + x1] - t[y1 * s + x0] + t[y0 * s + x0];
    }
    void stats(int64_t x, int64_t y, int64_t bw, int64_t bh, float* mean, float* sd) const {
        const int64_t s = w + 1;
        const double n = (double)(bw * bh);
        const double m = rect(sum, s, x, y, x + bw, y + bh) / n;
        const double var = rect(sumsq, s, x, y, x + bw, y + bh) / n - m * m;
        *mean = (float)m;
        *sd = (float)std::sqrt(std::max(var, 0.0));
    }
};

// ---------------------------------------------------------------------------------------------
// Validation helpers (validate.rs:133-170)
// ---------------------------------------------------------------------------------------------
// f32::total_cmp for non-NaN values (validate.rs:164): ascending, -0.0 before +0.0. The signed
// integer key of the bit pattern orders exactly so.
int32_t total_key(float f) {
    int32_t b;
    std::memcpy(&b, &f, sizeof b);
    return b ^ ((b >> 31) & 0x7fffffff);
}

float median(float* v, int n) {
    std::sort(v, v + n, [](float a, float b) { return total_key(a) < total_key(b); });
    if (n % 2 == 1) return v[n / 2];
    return 0.5f * (v[n / 2 - 1] + v[n / 2]);
}

int collect(const float* dx, const float* dy, const uint8_t* snap, int64_t ny, int64_t nx, int64_t ix,
            int64_t iy, int64_t radius, float* nu, float* nv) {
    int cnt = 0;
    const int64_t ylo = iy >= radius ? iy - radius : 0, yhi = std::min(iy + radius, ny - 1);
    const int64_t xlo = ix >= radius ? ix - radius : 0, xhi = std::min(ix + radius, nx - 1);
    for (int64_t y = ylo; y <= yhi; ++y)
        for (int64_t x = xlo; x <= xhi; ++x)
            if (!(x == ix && y == iy) && (snap[y * nx + x] & INVALID) == 0) {
                nu[cnt] = dx[y * nx + x];
                nv[cnt] = dy[y * nx + x];
                ++cnt;
            }
    return cnt;
}

float residual(float value, float* nb, int n, float eps) {
    const float med = median(nb, n);
    float dev[32];
    for (int i = 0; i < n; ++i) dev[i] = std::fabs(nb[i] - med);
    return std::fabs(value - med) / (median(dev, n) + eps);
}

int num_threads(int nthreads) {
#ifdef _OPENMP
    return nthreads > 0 ? nthreads : omp_get_max_threads();
#else
    (void)nthreads;
    return 1;
#endif
}

}  // namespace

extern "C" {

int orc_grid(int64_t height, int64_t width, int64_t window, float overlap, OrcGrid* g) {
    if (!(overlap >= 0.0f && overlap < 1.0f)) return ORC_ERR_CONFIG;
    if (window == 0 || window > width || window > height) return ORC_ERR_TOO_SMALL;
    const float st = std::round((float)window * (1.0f - overlap));  // round half away from zero
    int64_t step = st > 0.0f ? (int64_t)st : 0;
    step = std::max<int64_t>(step, 1);
    g->window = window;
    g->step = step;
    g->nx = (width - window) / step + 1;
    g->ny = (height - window) / step + 1;
    g->x0 = (width - window - (g->nx - 1) * step) / 2;
    g->y0 = (height - window - (g->ny - 1) * step) / 2;
    return ORC_OK;
}

void orc_u8_to_f32(const uint8_t* src, int64_t n, float* dst) {
    for (int64_t i = 0; i < n; ++i) dst[i] = (float)src[i] / 255.0f;
}

void orc_u16_to_f32(const uint16_t* src, int64_t n, float* dst) {
    for (int64_t i = 0; i < n; ++i) dst[i] = (float)src[i] / 65535.0f;
}

int64_t orc_percentile_clip_u16(uint16_t* codes, int64_t n, double percentile) {
    if (n <= 0) return 0;
    std::vector<int64_t> hist(65536, 0);
    for (int64_t i = 0; i < n; ++i) hist[codes[i]]++;
    double p = std::min(std::max(percentile, 0.0), 100.0);
    int64_t target = (int64_t)std::ceil(p / 100.0 * (double)n);
    if (target < 1) target = 1;
    int64_t acc = 0, clip = 65535;
    for (int64_t c = 0; c < 65536; ++c) {
        acc += hist[c];
        if (acc >= target) {
            clip = c;
            break;
        }
    }
    for (int64_t i = 0; i < n; ++i)
        if (codes[i] > clip) codes[i] = (uint16_t)clip;
    return clip;
}

void orc_background(const float* frames, int64_t count, int64_t npix, int mode, float* out) {
    if (count <= 0) return;
    std::memcpy(out, frames, sizeof(float) * npix);
    for (int64_t f = 1; f < count; ++f) {
        const float* fr = frames + f * npix;
        for (int64_t i = 0; i < npix; ++i) {
            if (mode == 0)
                out[i] = std::fmin(out[i], fr[i]);  // Rust f32::min ignores NaN like fmin
            else
                out[i] += fr[i];
        }
    }
    if (mode == 1)
        for (int64_t i = 0; i < npix; ++i) out[i] /= (float)count;
}

void orc_gaussian_blur(const float* src, int64_t h, int64_t w, float sigma, float* out) {
    // preprocess.rs:161-195
    const int64_t radius = (int64_t)std::max(std::ceil(3.0f * sigma), 1.0f);
    std::vector<float> k;
    for (int64_t i = -radius; i <= radius; ++i)
        k.push_back(std::exp(-(float)(i * i) / (2.0f * sigma * sigma)));
    float total = 0.0f;
    for (float v : k) total += v;
    for (float& v : k) v /= total;
    std::vector<float> tmp(h * w);
#pragma omp parallel for schedule(static)
    for (int64_t y = 0; y < h; ++y) {
        const float* row = src + y * w;
        for (int64_t x = 0; x < w; ++x) {
            float s = -0.0f;
            for (size_t j = 0; j < k.size(); ++j) {
                int64_t sx = std::min(std::max(x + (int64_t)j - radius, (int64_t)0), w - 1);
                s += k[j] * row[sx];
            }
            tmp[y * w + x] = s;
        }
    }
#pragma omp parallel for schedule(static)
    for (int64_t y = 0; y < h; ++y) {
        float* o = out + y * w;
        for (int64_t x = 0; x < w; ++x) o[x] = 0.0f;
        for (size_t j = 0; j < k.size(); ++j) {
            int64_t sy = std::min(std::max(y + (int64_t)j - radius, (int64_t)0), h - 1);
            const float* row = tmp.data() + sy * w;
            for (int64_t x = 0; x < w; ++x) o[x] += k[j] * row[x];
        }
    }
}

void orc_local_normalize(const float* src, int64_t h, int64_t w, int64_t radius, float eps, float* out) {
    // preprocess.rs:199-216
    Integral ii(src, h, w);
#pragma omp parallel for schedule(static)
    for (int64_t y = 0; y < h; ++y) {
        const int64_t y0 = y >= radius ? y - radius : 0, y1 = std::min(y + radius + 1, h);
        for (int64_t x = 0; x < w; ++x) {
            const int64_t x0 = x >= radius ? x - radius : 0, x1 = std::min(x + radius + 1, w);
            float mean, sd;
            ii.stats(x0, y0, x1 - x0, y1 - y0, &mean, &sd);
            out[y * w + x] = (src[y * w + x] - mean) / (sd + eps);
        }
    }
}

void orc_prepare(const float* raw, const float* background, int64_t h, int64_t w, float smooth_sigma,
                 int64_t normalize_radius, float normalize_eps, float* image_out, float* base_out) {
    // preprocess.rs:138-158
    std::vector<float> base(raw, raw + h * w);
    if (background)
        for (int64_t i = 0; i < h * w; ++i) base[i] = std::fmax(base[i] - background[i], 0.0f);
    if (base_out) std::memcpy(base_out, base.data(), sizeof(float) * h * w);
    std::vector<float> image(h * w);
    if (smooth_sigma > 0.0f)
        orc_gaussian_blur(base.data(), h, w, smooth_sigma, image.data());
    else
        image = base;
    if (normalize_radius > 0) {
        std::vector<float> tmp(h * w);
        orc_local_normalize(image.data(), h, w, normalize_radius, normalize_eps, tmp.data());
        image.swap(tmp);
    }
    std::memcpy(image_out, image.data(), sizeof(float) * h * w);
}

void orc_box_stats(const float* frame, int64_t h, int64_t w, int64_t bx, int64_t by, int64_t bw,
                   int64_t bh, float* mean, float* sd) {
    Integral ii(frame, h, w);
    ii.stats(bx, by, bw, bh, mean, sd);
}

}  // extern "C"

namespace {

// VectorField::sample (field.rs:56-81): bilinear on the predictor grid, clamped, NaN skipped.
void sample_pred(const OrcGrid* pg, const float* pdx, const float* pdy, float x, float y, float* px, float* py) {
    *px = 0.0f;
    *py = 0.0f;
    const float fx = clampf((x - center(pg->x0, 0, pg->step, pg->window)) / (float)pg->step, 0.0f, (float)(pg->nx - 1));
    const float fy = clampf((y - center(pg->y0, 0, pg->step, pg->window)) / (float)pg->step, 0.0f, (float)(pg->ny - 1));
    const int64_t jx = (int64_t)std::floor(fx), jy = (int64_t)std::floor(fy);
    const float tx = fx - (float)jx, ty = fy - (float)jy;
    const int64_t jx1 = std::min(jx + 1, pg->nx - 1), jy1 = std::min(jy + 1, pg->ny - 1);
    const int64_t rr[4] = {jy, jy, jy1, jy1};
    const int64_t cc[4] = {jx, jx1, jx, jx1};
    const float ww[4] = {(1.0f - tx) * (1.0f - ty), tx * (1.0f - ty), (1.0f - tx) * ty, tx * ty};
    float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f;
    for (int j = 0; j < 4; ++j) {
        const float u = pdx[rr[j] * pg->nx + cc[j]], v = pdy[rr[j] * pg->nx + cc[j]];
        if (ww[j] > 0.0f && std::isfinite(u) && std::isfinite(v)) {
            a0 = a0 + ww[j] * u;
            a1 = a1 + ww[j] * v;
            a2 = a2 + ww[j];
        }
    }
    if (a2 > 0.0f) {
        *px = a0 / a2;
        *py = a1 / a2;
    }
}

// Deformed-window helpers (see piv_oracle.h).
// Base position of a deformed window: its zero-shift origin under the placement clamp
// (multipass.rs:207-208, 224-231 with shift 0), i.e. the grid origin clamped to w - n - 1.
int64_t deform_base(int64_t origin, int64_t extent, int64_t n) {
    return std::min(std::max<int64_t>(origin, 0), std::max<int64_t>(extent - n - 1, 0));
}

template <class T>
T blend(const float* c, int k, T u, T v) {
    const T w00 = ((T)1 - u) * ((T)1 - v), w10 = u * ((T)1 - v), w01 = ((T)1 - u) * v, w11 = u * v;
    return w00 * (T)c[k] + w10 * (T)c[2 + k] + w01 * (T)c[4 + k] + w11 * (T)c[6 + k];
}

template <class T>
T bilinear_clamped(const float* img, int64_t h, int64_t w, T px, T py) {
    px = std::min(std::max(px, (T)0), (T)(w - 1));
    py = std::min(std::max(py, (T)0), (T)(h - 1));
    int64_t ix = (int64_t)std::floor(px), iy = (int64_t)std::floor(py);
    ix = std::min(ix, std::max<int64_t>(w - 2, 0));
    iy = std::min(iy, std::max<int64_t>(h - 2, 0));
    const T tx = px - (T)ix, ty = py - (T)iy;
    const int64_t ix1 = std::min(ix + 1, w - 1), iy1 = std::min(iy + 1, h - 1);
    const T w00 = ((T)1 - tx) * ((T)1 - ty), w01 = tx * ((T)1 - ty), w10 = ((T)1 - tx) * ty, w11 = tx * ty;
    return w00 * (T)img[iy * w + ix] + w01 * (T)img[iy * w + ix1] + w10 * (T)img[iy1 * w + ix] +
           w11 * (T)img[iy1 * w + ix1];
}

// Window sample of the deformed window (sign -1: frame A, +1: frame B), then mean removal and
// energy as load_window (correlate.rs:203-209).
template <class T>
double load_window_deform(const float* img, int64_t h, int64_t w, int64_t x0, int64_t y0, int64_t n,
                          const float* corners, T sign, T* dst) {
    for (int64_t r = 0; r < n; ++r)
        for (int64_t c = 0; c < n; ++c) {
            const T u = (T)c / (T)(n - 1), v = (T)r / (T)(n - 1);
            const T px = (T)(x0 + c) + sign * ((T)0.5 * blend<T>(corners, 0, u, v));
            const T py = (T)(y0 + r) + sign * ((T)0.5 * blend<T>(corners, 1, u, v));
            dst[r * n + c] = bilinear_clamped<T>(img, h, w, px, py);
        }
    double s = 0.0;
    for (int64_t i = 0; i < n * n; ++i) s += (double)dst[i];
    const double mean = s / (double)(n * n);
    const T mf = (T)mean;
    double energy = 0.0;
    for (int64_t i = 0; i < n * n; ++i) {
        dst[i] -= mf;
        energy += (double)dst[i] * (double)dst[i];
    }
    return energy;
}

}  // namespace

extern "C" {

void orc_place(const OrcGrid* g, int64_t h, int64_t w, const OrcGrid* pg, const float* pdx,
               const float* pdy, float* origins) {
    // multipass.rs:204-231, field.rs:56-81
    const int64_t n = g->window;
    const float max_x = (float)std::max<int64_t>(w - n - 1, 0);
    const float max_y = (float)std::max<int64_t>(h - n - 1, 0);
    for (int64_t iy = 0; iy < g->ny; ++iy)
        for (int64_t ix = 0; ix < g->nx; ++ix) {
            float px = 0.0f, py = 0.0f;
            if (pg && pdx && pdy)
                sample_pred(pg, pdx, pdy, center(g->x0, ix, g->step, g->window), center(g->y0, iy, g->step, g->window),
                            &px, &py);
            auto place = [](int64_t origin, float shift, float mx, float* a, float* b) {
                const float s = clampf(shift, -mx, mx);
                const float a0 = clampf((float)origin - s / 2.0f, std::fmax(-s, 0.0f), std::fmin(mx - s, mx));
                *a = a0;
                *b = a0 + s;
            };
            float* o = origins + 4 * (iy * g->nx + ix);
            place(g->x0 + ix * g->step, px, max_x, &o[0], &o[2]);
            place(g->y0 + iy * g->step, py, max_y, &o[1], &o[3]);
        }
}

void orc_correlate_pass(const float* image_a, const float* image_b, const float* base_a,
                        const float* base_b, int64_t h, int64_t w, int64_t n, int64_t ncells,
                        const float* origins, float min_mean, float min_std, int mode, int nthreads,
                        float* dx, float* dy, float* ppr, uint8_t* flags) {
    // multipass.rs:210-259
    Integral sa(base_a, h, w), sb(base_b, h, w);
    const int nt = num_threads(nthreads);
#pragma omp parallel num_threads(nt)
    {
        Workspace<float> wsf(mode == ORC_REF ? n : 2);
        Workspace<double> wsd(mode == ORC_FP64 ? n : 2);
#pragma omp for schedule(dynamic, 16)
        for (int64_t k = 0; k < ncells; ++k) {
            const float* o = origins + 4 * k;
            const float ax = o[0], ay = o[1], bx = o[2], by = o[3];
            auto has_signal = [&](const Integral& s, float x, float y) {
                float mean, sd;
                s.stats((int64_t)std::round(x), (int64_t)std::round(y), n, n, &mean, &sd);
                return mean >= min_mean && sd >= min_std;
            };
            bool ok = has_signal(sa, ax, ay) && has_signal(sb, bx, by);
            float pk[4];
            if (ok) {
                if (mode == ORC_REF) {
                    ok = wsf.plane(image_a, w, ax, ay, image_b, w, bx, by);
                    if (ok) find_peak_t<float>(wsf.corr.data(), n, pk);
                } else {
                    ok = wsd.plane(image_a, w, ax, ay, image_b, w, bx, by);
                    if (ok) {
                        // Peak and assembly in f64, rounded once.
                        double pd[4];
                        find_peak_t<double>(wsd.corr.data(), n, pd);
                        dx[k] = (float)((double)bx - (double)ax + pd[0]);
                        dy[k] = (float)((double)by - (double)ay + pd[1]);
                        ppr[k] = (float)pd[3];
                        flags[k] = 0;
                        continue;
                    }
                }
            }
            if (!ok) {
                dx[k] = NAN;
                dy[k] = NAN;
                ppr[k] = 0.0f;
                flags[k] = NO_SIGNAL;
            } else {
                dx[k] = bx - ax + pk[0];
                dy[k] = by - ay + pk[1];
                ppr[k] = pk[3];
                flags[k] = 0;
            }
        }
    }
}

void orc_place_deform(const OrcGrid* g, int64_t h, int64_t w, const OrcGrid* pg, const float* pdx,
                      const float* pdy, float* origins, float* corners) {
    orc_place(g, h, w, pg, pdx, pdy, origins);
    const int64_t n = g->window;
    for (int64_t iy = 0; iy < g->ny; ++iy)
        for (int64_t ix = 0; ix < g->nx; ++ix) {
            float* c = corners + 8 * (iy * g->nx + ix);
            const float x0 = (float)deform_base(g->x0 + ix * g->step, w, n);
            const float y0 = (float)deform_base(g->y0 + iy * g->step, h, n);
            const float xs[4] = {x0, x0 + (float)(n - 1), x0, x0 + (float)(n - 1)};
            const float ys[4] = {y0, y0, y0 + (float)(n - 1), y0 + (float)(n - 1)};
            for (int j = 0; j < 4; ++j) {
                c[2 * j] = 0.0f;
                c[2 * j + 1] = 0.0f;
                if (pg && pdx && pdy) sample_pred(pg, pdx, pdy, xs[j], ys[j], &c[2 * j], &c[2 * j + 1]);
            }
        }
}

void orc_correlate_pass_deform(const float* image_a, const float* image_b, const float* base_a,
                               const float* base_b, int64_t h, int64_t w, const OrcGrid* g,
                               const float* origins, const float* corners, float min_mean, float min_std,
                               int mode, int nthreads, float* dx, float* dy, float* ppr, uint8_t* flags) {
    Integral sa(base_a, h, w), sb(base_b, h, w);
    const int64_t n = g->window, ncells = g->nx * g->ny;
    const int nt = num_threads(nthreads);
#pragma omp parallel num_threads(nt)
    {
        Workspace<float> wsf(mode == ORC_REF ? n : 2);
        Workspace<double> wsd(mode == ORC_FP64 ? n : 2);
#pragma omp for schedule(dynamic, 16)
        for (int64_t k = 0; k < ncells; ++k) {
            const float* o = origins + 4 * k;
            const float* c = corners + 8 * k;
            const int64_t x0 = deform_base(g->x0 + (k % g->nx) * g->step, w, n);
            const int64_t y0 = deform_base(g->y0 + (k / g->nx) * g->step, h, n);
            auto has_signal = [&](const Integral& s, float x, float y) {
                float mean, sd;
                s.stats((int64_t)std::round(x), (int64_t)std::round(y), n, n, &mean, &sd);
                return mean >= min_mean && sd >= min_std;
            };
            bool ok = has_signal(sa, o[0], o[1]) && has_signal(sb, o[2], o[3]);
            if (ok) {
                if (mode == ORC_REF) {
                    const double ea = load_window_deform<float>(image_a, h, w, x0, y0, n, c, -1.0f, wsf.a.data());
                    const double eb = load_window_deform<float>(image_b, h, w, x0, y0, n, c, 1.0f, wsf.b.data());
                    ok = wsf.finish(ea, eb);
                    if (ok) {
                        float pk[4];
                        find_peak_t<float>(wsf.corr.data(), n, pk);
                        dx[k] = blend<float>(c, 0, 0.5f, 0.5f) + pk[0];
                        dy[k] = blend<float>(c, 1, 0.5f, 0.5f) + pk[1];
                        ppr[k] = pk[3];
                    }
                } else {
                    const double ea = load_window_deform<double>(image_a, h, w, x0, y0, n, c, -1.0, wsd.a.data());
                    const double eb = load_window_deform<double>(image_b, h, w, x0, y0, n, c, 1.0, wsd.b.data());
                    ok = wsd.finish(ea, eb);
                    if (ok) {
                        double pd[4];
                        find_peak_t<double>(wsd.corr.data(), n, pd);
                        dx[k] = (float)(blend<double>(c, 0, 0.5, 0.5) + pd[0]);
                        dy[k] = (float)(blend<double>(c, 1, 0.5, 0.5) + pd[1]);
                        ppr[k] = (float)pd[3];
                    }
                }
            }
            if (!ok) {
                dx[k] = NAN;
                dy[k] = NAN;
                ppr[k] = 0.0f;
                flags[k] = NO_SIGNAL;
            } else {
                flags[k] = 0;
            }
        }
    }
}

int orc_correlation_plane(const float* a, int64_t ha, int64_t wa, float ax, float ay, const float* b,
                          int64_t hb, int64_t wb, float bx, float by, int64_t n, int mode, float* plane) {
    (void)ha;
    (void)hb;
    if (mode == ORC_REF) {
        Workspace<float> ws(n);
        if (!ws.plane(a, wa, ax, ay, b, wb, bx, by)) return 0;
        std::memcpy(plane, ws.corr.data(), sizeof(float) * n * n);
    } else {
        Workspace<double> ws(n);
        if (!ws.plane(a, wa, ax, ay, b, wb, bx, by)) return 0;
        for (int64_t i = 0; i < n * n; ++i) plane[i] = (float)ws.corr[i];
    }
    return 1;
}

int orc_correlate_window(const float* a, int64_t ha, int64_t wa, float ax, float ay, const float* b,
                         int64_t hb, int64_t wb, float bx, float by, int64_t n, int mode, float* peak) {
    (void)ha;
    (void)hb;
    if (mode == ORC_REF) {
        Workspace<float> ws(n);
        if (!ws.plane(a, wa, ax, ay, b, wb, bx, by)) return 0;
        find_peak_t<float>(ws.corr.data(), n, peak);
    } else {
        Workspace<double> ws(n);
        if (!ws.plane(a, wa, ax, ay, b, wb, bx, by)) return 0;
        double pd[4];
        find_peak_t<double>(ws.corr.data(), n, pd);
        for (int i = 0; i < 4; ++i) peak[i] = (float)pd[i];
    }
    return 1;
}

double orc_load_window(const float* img, int64_t h, int64_t w, float x, float y, int64_t n, float* dst) {
    (void)h;
    return load_window_f32(img, w, x, y, n, dst);
}

void orc_find_peak(const float* corr, int64_t n, float* peak) { find_peak_t<float>(corr, n, peak); }

void orc_validate(float* dx, float* dy, const float* ppr, uint8_t* flags, int64_t ny, int64_t nx,
                  float ppr_threshold, float median_threshold, float median_eps, int replace,
                  float max_displacement, OrcSummary* summary) {
    // validate.rs:51-130
    OrcSummary s = {0, 0, 0, 0, 0};
    const int64_t cnt = ny * nx;
    for (int64_t i = 0; i < cnt; ++i) {
        if (flags[i] & NO_SIGNAL) {
            s.no_signal++;
            continue;
        }
        if (std::hypot(dx[i], dy[i]) > max_displacement) {
            flags[i] |= OUT_OF_RANGE;
            s.out_of_range++;
        }
        if (ppr[i] < ppr_threshold) {
            flags[i] |= LOW_PPR;
            s.low_ppr++;
        }
    }
    std::vector<uint8_t> snap(flags, flags + cnt);
    float nu[32], nv[32];
    for (int64_t iy = 0; iy < ny; ++iy)
        for (int64_t ix = 0; ix < nx; ++ix) {
            if (snap[iy * nx + ix] & INVALID) continue;
            const int c = collect(dx, dy, snap.data(), ny, nx, ix, iy, 1, nu, nv);
            if (c < 2) continue;
            const float ru = residual(dx[iy * nx + ix], nu, c, median_eps);
            const float rv = residual(dy[iy * nx + ix], nv, c, median_eps);
            if (std::sqrt(ru * ru + rv * rv) > median_threshold) {
                flags[iy * nx + ix] |= MEDIAN_OUTLIER;
                s.median_outliers++;
            }
        }
    if (replace) {
        snap.assign(flags, flags + cnt);
        for (int64_t iy = 0; iy < ny; ++iy)
            for (int64_t ix = 0; ix < nx; ++ix) {
                const uint8_t f = snap[iy * nx + ix];
                if (!((f & NO_SIGNAL) == 0 && (f & INVALID) != 0)) continue;
                bool done = false;
                for (int64_t radius = 1; radius <= 2; ++radius) {
                    const int c = collect(dx, dy, snap.data(), ny, nx, ix, iy, radius, nu, nv);
                    if (c > 0) {
                        dx[iy * nx + ix] = median(nu, c);
                        dy[iy * nx + ix] = median(nv, c);
                        flags[iy * nx + ix] |= REPLACED;
                        s.replaced++;
                        done = true;
                        break;
                    }
                }
                if (!done) {
                    dx[iy * nx + ix] = NAN;
                    dy[iy * nx + ix] = NAN;
                }
            }
    }
    if (summary) *summary = s;
}

int orc_check_config(const OrcConfig* cfg) {
    // multipass.rs:91-119
    if (cfg->n_windows <= 0) return ORC_ERR_CONFIG;
    for (int i = 0; i < cfg->n_windows; ++i)
        if (cfg->windows[i] < 8 || cfg->windows[i] % 2 != 0) return ORC_ERR_CONFIG;
    if (!(cfg->overlap >= 0.0f && cfg->overlap < 1.0f)) return ORC_ERR_CONFIG;
    if (cfg->final_iterations < 1) return ORC_ERR_CONFIG;
    return ORC_OK;
}

int orc_num_passes(const OrcConfig* cfg) { return cfg->n_windows + cfg->final_iterations - 1; }

int orc_analyze(const OrcConfig* cfg, const float* image_a, const float* image_b, const float* base_a,
                const float* base_b, int64_t h, int64_t w, int mode, int nthreads, float* final_dx,
                float* final_dy, float* final_ppr, uint8_t* final_flags, OrcSummary* summary,
                float* trace_origins, float* trace_raw_dx, float* trace_raw_dy, float* trace_raw_ppr,
                uint8_t* trace_raw_flags, float* trace_dx, float* trace_dy, float* trace_ppr,
                uint8_t* trace_flags) {
    // multipass.rs:152-192
    int st = orc_check_config(cfg);
    if (st) return st;
    const int npass = orc_num_passes(cfg);
    std::vector<float> pdx, pdy;
    OrcGrid pg{};
    bool have_pred = false;
    int64_t toff = 0;
    for (int p = 0; p < npass; ++p) {
        const int64_t win = p < cfg->n_windows ? cfg->windows[p] : cfg->windows[cfg->n_windows - 1];
        OrcGrid g;
        st = orc_grid(h, w, win, cfg->overlap, &g);
        if (st) return st;
        const int64_t cells = g.nx * g.ny;
        std::vector<float> origins(4 * cells), dx(cells), dy(cells), ppr(cells);
        std::vector<uint8_t> fl(cells);
        if (cfg->deform && have_pred) {
            std::vector<float> corners(8 * cells);
            orc_place_deform(&g, h, w, &pg, pdx.data(), pdy.data(), origins.data(), corners.data());
            orc_correlate_pass_deform(image_a, image_b, base_a, base_b, h, w, &g, origins.data(), corners.data(),
                                      cfg->min_mean, cfg->min_std, mode, nthreads, dx.data(), dy.data(), ppr.data(),
                                      fl.data());
        } else {
            orc_place(&g, h, w, have_pred ? &pg : nullptr, have_pred ? pdx.data() : nullptr,
                      have_pred ? pdy.data() : nullptr, origins.data());
            orc_correlate_pass(image_a, image_b, base_a, base_b, h, w, win, cells, origins.data(),
                               cfg->min_mean, cfg->min_std, mode, nthreads, dx.data(), dy.data(), ppr.data(),
                               fl.data());
        }
        if (trace_origins) std::memcpy(trace_origins + 4 * toff, origins.data(), sizeof(float) * 4 * cells);
        if (trace_raw_dx) std::memcpy(trace_raw_dx + toff, dx.data(), sizeof(float) * cells);
        if (trace_raw_dy) std::memcpy(trace_raw_dy + toff, dy.data(), sizeof(float) * cells);
        if (trace_raw_ppr) std::memcpy(trace_raw_ppr + toff, ppr.data(), sizeof(float) * cells);
        if (trace_raw_flags) std::memcpy(trace_raw_flags + toff, fl.data(), cells);
        OrcSummary s;
        orc_validate(dx.data(), dy.data(), ppr.data(), fl.data(), g.ny, g.nx, cfg->ppr_threshold,
                     cfg->median_threshold, cfg->median_eps, cfg->replace, (float)cfg->windows[0] / 2.0f, &s);
        if (trace_dx) std::memcpy(trace_dx + toff, dx.data(), sizeof(float) * cells);
        if (trace_dy) std::memcpy(trace_dy + toff, dy.data(), sizeof(float) * cells);
        if (trace_ppr) std::memcpy(trace_ppr + toff, ppr.data(), sizeof(float) * cells);
        if (trace_flags) std::memcpy(trace_flags + toff, fl.data(), cells);
        toff += cells;
        if (p == npass - 1) {
            if (final_dx) std::memcpy(final_dx, dx.data(), sizeof(float) * cells);
            if (final_dy) std::memcpy(final_dy, dy.data(), sizeof(float) * cells);
            if (final_ppr) std::memcpy(final_ppr, ppr.data(), sizeof(float) * cells);
            if (final_flags) std::memcpy(final_flags, fl.data(), cells);
            if (summary) *summary = s;
        }
        pdx.swap(dx);
        pdy.swap(dy);
        pg = g;
        have_pred = true;
    }
    return ORC_OK;
}

// ---------------------------------------------------------------------------------------------
// Post-processing of validated fields (the path's next components).
// ---------------------------------------------------------------------------------------------
void orc_usable(const float* dx, const uint8_t* flags, int64_t n, uint8_t* usable) {
    // flow.rs:13-17: finite and accepted, or interpolated (REPLACED)
    for (int64_t i = 0; i < n; ++i)
        usable[i] = std::isfinite(dx[i]) && ((flags[i] & INVALID) == 0 || (flags[i] & REPLACED) != 0);
}

extern "C++" {
namespace {
// flowstats.rs:28-39: central difference where both neighbours are usable, one-sided otherwise.
template <class At>
bool derivative(int64_t i, int64_t n, float h, At at, float* out) {
    float c, l, r;
    if (!at(i, &c)) return false;
    const bool hl = i >= 1 && at(i - 1, &l);
    const bool hr = i + 1 < n && at(i + 1, &r);
    if (hl && hr) *out = (r - l) / (2.0f * h);
    else if (hl) *out = (c - l) / h;
    else if (hr) *out = (r - c) / h;
    else return false;
    return true;
}
}  // namespace
}  // extern "C++"

void orc_vorticity(const float* u, const float* v, const uint8_t* usable, int64_t ny, int64_t nx, float step,
                   float* w) {
    // flowstats.rs:44-64: w = du/dy - dv/dx (image axes), NaN where either derivative is missing
    auto get = [&](const float* a, int64_t iy, int64_t ix, float* o) {
        const float x = a[iy * nx + ix];
        if (!(usable[iy * nx + ix] && std::isfinite(x))) return false;
        *o = x;
        return true;
    };
    for (int64_t iy = 0; iy < ny; ++iy)
        for (int64_t ix = 0; ix < nx; ++ix) {
            float a, b;
            const bool ha = derivative(iy, ny, step, [&](int64_t j, float* o) { return get(u, j, ix, o); }, &a);
            const bool hb = derivative(ix, nx, step, [&](int64_t j, float* o) { return get(v, iy, j, o); }, &b);
            w[iy * nx + ix] = (ha && hb) ? a - b : NAN;
        }
}

void orc_flow_stats(const float* u, const float* v, const uint8_t* usable, int64_t ny, int64_t nx, float step,
                    OrcFlowStats* out) {
    // flowstats.rs:67-101
    std::vector<float> w((size_t)(ny * nx));
    orc_vorticity(u, v, usable, ny, nx, step, w.data());
    double ws = 0.0, wa = 0.0, e = 0.0;
    int64_t nw = 0, n = 0;
    for (float x : w)
        if (std::isfinite(x)) {
            ws += (double)x;
            wa += (double)std::fabs(x);
            ++nw;
        }
    for (int64_t i = 0; i < ny * nx; ++i)
        if (usable[i] && std::isfinite(u[i]) && std::isfinite(v[i])) {
            e += 0.5 * ((double)u[i] * (double)u[i] + (double)v[i] * (double)v[i]);
            ++n;
        }
    auto mean = [](double s, int64_t k) { return k > 0 ? (float)(s / (double)k) : NAN; };
    out->vorticity_mean = mean(ws, nw);
    out->vorticity_abs_mean = mean(wa, nw);
    out->ke_mean = mean(e, n);
    out->ke_sum = (float)(e * std::pow((double)step, 2.0));
    out->coverage = (float)n / (float)std::max<int64_t>(ny * nx, 1);
    out->n_usable = n;
    out->n_vorticity = nw;
}

void orc_pair_stats(const float* dx, const float* dy, const uint8_t* flags, int64_t ny, int64_t nx, int64_t step,
                    double dt_s, OrcFlowStats* out) {
    // flow.rs:20-36: px/s from px with k = (1 / dt) as f32
    const int64_t n = ny * nx;
    const float k = (float)(1.0 / dt_s);
    std::vector<float> u((size_t)n), v((size_t)n);
    std::vector<uint8_t> us((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        u[i] = dx[i] * k;
        v[i] = dy[i] * k;
    }
    orc_usable(dx, flags, n, us.data());
    orc_flow_stats(u.data(), v.data(), us.data(), ny, nx, (float)step, out);
}

extern "C++" {
namespace {
float mean_seq(const float* v, int n) {
    float s = 0.0f;
    for (int i = 0; i < n; ++i) s += v[i];
    return s / (float)n;
}
float median_sorted(float* v, int n) {
    std::sort(v, v + n, [](float a, float b) { return a < b; });
    return (n % 2 == 1) ? v[n / 2] : 0.5f * (v[n / 2 - 1] + v[n / 2]);
}
}  // namespace
}  // extern "C++"

int orc_temporal_offsets(int32_t window, const int32_t* leave_out, int32_t n_leave, int32_t* offsets) {
    // smooth.rs:59-73: centre unless left out, then half offsets each side skipping left-out ones
    auto left = [&](int32_t o) {
        for (int32_t i = 0; i < n_leave; ++i)
            if (leave_out[i] == o) return true;
        return false;
    };
    int c = 0;
    if (!left(0)) offsets[c++] = 0;
    const int32_t half = window / 2;
    for (int32_t sign : {-1, 1}) {
        int32_t k = 1, taken = 0;
        while (taken < half) {
            if (!left(sign * k)) {
                offsets[c++] = sign * k;
                ++taken;
            }
            ++k;
        }
    }
    return c;
}

void orc_temporal(const float* dx, const float* dy, const uint8_t* usable, const uint8_t* gate, int64_t nt,
                  int64_t ny, int64_t nx, int32_t median, int32_t window, int32_t min_support, const int32_t* leave_out,
                  int32_t n_leave, float* out_dx, float* out_dy, uint16_t* support) {
    // smooth.rs:44-128
    std::vector<int32_t> off((size_t)window + 1);
    const int no = orc_temporal_offsets(window, leave_out, n_leave, off.data());
    const int64_t plane = ny * nx;
    std::vector<float> bu((size_t)no), bv((size_t)no);
    for (int64_t t = 0; t < nt; ++t)
        for (int64_t k = 0; k < plane; ++k) {
            const int64_t o = t * plane + k;
            out_dx[o] = NAN;
            out_dy[o] = NAN;
            support[o] = 0;
            if (!gate[o]) continue;
            int c = 0;
            for (int j = 0; j < no; ++j) {
                const int64_t s = t + off[j];
                if (s < 0 || s >= nt || !usable[s * plane + k]) continue;
                bu[c] = dx[s * plane + k];
                bv[c] = dy[s * plane + k];
                ++c;
            }
            support[o] = (uint16_t)c;
            if (c >= std::max(min_support, 1)) {
                out_dx[o] = median ? median_sorted(bu.data(), c) : mean_seq(bu.data(), c);
                out_dy[o] = median ? median_sorted(bv.data(), c) : mean_seq(bv.data(), c);
            }
        }
}

int orc_spatial_kernel(float sigma, int32_t leave_out, float* weights, float* full, float* total) {
    // smooth.rs:143-166: radius max(ceil(2.5 sigma), 1); weights exp(-(i^2+j^2) / (2 sigma^2))
    const int r = std::max((int)std::ceil(2.5f * sigma), 1);
    const int d = 2 * r + 1;
    float f = 0.0f, t = 0.0f;
    for (int j = -r; j <= r; ++j)
        for (int i = -r; i <= r; ++i) {
            const float w = std::exp(-((float)(i * i + j * j)) / (2.0f * sigma * sigma));
            if (weights) weights[(j + r) * d + (i + r)] = w;
        }
    for (int j = -r; j <= r; ++j)
        for (int i = -r; i <= r; ++i) {
            const float w = std::exp(-((float)(i * i + j * j)) / (2.0f * sigma * sigma));
            const bool ex = leave_out >= 0 && std::max(std::abs(i), std::abs(j)) <= leave_out;
            if (!ex) f += w;
            t += w;
        }
    *full = f;
    *total = t;
    return r;
}

void orc_spatial(const float* dx, const float* dy, const uint8_t* gate, int64_t nt, int64_t ny, int64_t nx,
                 float sigma, float min_weight, int32_t leave_out, float* out_dx, float* out_dy, uint16_t* support) {
    // smooth.rs:130-207: normalized convolution, NaN neighbours skipped
    float full, total;
    const int r = orc_spatial_kernel(sigma, leave_out, nullptr, &full, &total);
    const int d = 2 * r + 1;
    std::vector<float> kern((size_t)(d * d));
    orc_spatial_kernel(sigma, leave_out, kern.data(), &full, &total);
    const int64_t plane = ny * nx;
    for (int64_t i = 0; i < nt * plane; ++i) {
        out_dx[i] = NAN;
        out_dy[i] = NAN;
        support[i] = 0;
    }
    if (full < 0.5f * total) return;
    for (int64_t t = 0; t < nt; ++t)
        for (int64_t y = 0; y < ny; ++y)
            for (int64_t x = 0; x < nx; ++x) {
                const int64_t o = t * plane + y * nx + x;
                if (!gate[o]) continue;
                float su = 0.0f, sv = 0.0f, sw = 0.0f;
                int n = 0;
                for (int j = -r; j <= r; ++j) {
                    const int64_t yy = y + j;
                    if (yy < 0 || yy >= ny) continue;
                    for (int i = -r; i <= r; ++i) {
                        const int64_t xx = x + i;
                        if (xx < 0 || xx >= nx || (leave_out >= 0 && std::max(std::abs(i), std::abs(j)) <= leave_out))
                            continue;
                        const float a = dx[t * plane + yy * nx + xx], b = dy[t * plane + yy * nx + xx];
                        if (std::isfinite(a) && std::isfinite(b)) {
                            const float w = kern[(j + r) * d + (i + r)];
                            su += w * a;
                            sv += w * b;
                            sw += w;
                            ++n;
                        }
                    }
                }
                support[o] = (uint16_t)n;
                if (sw >= min_weight * full && sw > 0.0f) {
                    out_dx[o] = su / sw;
                    out_dy[o] = sv / sw;
                }
            }
}

uint64_t orc_splitmix_next(uint64_t* state) {
    // synthetic.rs:20-26
    *state += 0x9E3779B97F4A7C15ull;
    uint64_t z = *state;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

}  // extern "C"
