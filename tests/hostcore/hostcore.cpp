// Host build of device arithmetic of libpocean_b200 (test harness only): the exact constant divisions, the
// plane-index division and the one-pass column remap, compiled with g++ -ffp-contract=off so the tests can check them on the CPU against IEEE
// division and against the oracle.  Never linked into the product.
#include <cmath>
#include <cstdint>
#include <cstring>

#include "../../pyocean_b200/csrc/exactdiv.cuh"
#include "../../pyocean_b200/csrc/planediv.cuh"
#include "../../pyocean_b200/csrc/remap_core.cuh"

namespace {

uint64_t splitmix(uint64_t& s)
{
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

double bits(uint64_t u)
{
    double d;
    std::memcpy(&d, &u, 8);
    return d;
}

bool same(double a, double b)
{
    uint64_t x, y;
    std::memcpy(&x, &a, 8);
    std::memcpy(&y, &b, 8);
    return x == y || (std::isnan(a) && std::isnan(b));
}

struct HostIO {
    const double* h;
    const double* ht_;
    const double* u[4];
    double* o[4];
    double hs(int k) const { return h[k]; }
    double ht(int k) const { return ht_[k]; }
    double f(int m, int k) const { return u[m][k]; }
    void put(int m, int k, double v) { o[m][k] = v; }
};

}  // namespace

extern "C" {

// Mismatches of plane_div(p, plane_magic(nt)) against p / nt over every plane index 0 <= p < 65536, for the
// divisors nts[0..n).
long long check_plane_div(const int* nts, long long n)
{
    long long bad = 0;
    for (long long q = 0; q < n; ++q) {
        const int nt = nts[q];
        const unsigned m = po::plane_magic(nt);
        for (int p = 0; p < 65536; ++p) bad += po::plane_div(p, m) != p / nt;
    }
    return bad;
}

// Number of arguments x among n random bit patterns (every exponent) and n random values of ordinary magnitude
// for which div3_exact / div6_exact differ from IEEE division; mismatch examples go to bad[0..1].
long long check_exactdiv(long long n, unsigned long long seed, double* bad)
{
    uint64_t s = seed;
    long long fails = 0;
    for (long long t = 0; t < 2 * n; ++t) {
        double x = t < n ? bits(splitmix(s)) : ((double)(splitmix(s) >> 11) * 0x1p-53 - 0.5) * 1e4;
        if (!same(po::div3_exact(x), x / 3.0)) { if (!fails) bad[0] = x; ++fails; }
        if (!same(po::div6_exact(x), x / 6.0)) { if (!fails) bad[1] = x; ++fails; }
    }
    return fails;
}

// Edge values of the division check: each x of xs compared, returns the mismatch count.
long long check_exactdiv_list(const double* xs, long long n)
{
    long long fails = 0;
    for (long long t = 0; t < n; ++t) {
        const double x = xs[t];
        fails += !same(po::div3_exact(x), x / 3.0);
        fails += !same(po::div6_exact(x), x / 6.0);
    }
    return fails;
}

// One-pass remap of nf (1..2) fields of one column (the device sweep, on the host).  Returns 0, or 1 when the
// column is outside the sweep's domain (dry, or a negative / NaN target thickness) and nothing was written.
int remap_stream_column(const double* h_src, const double* f_src, int n0, const double* h_tgt, int n1, int nf,
                        int scheme, double* out)
{
    int n_active = 0, last = -1;
    for (int k = 0; k < n0; ++k)
        if (h_src[k] > 0.0) { ++n_active; last = k; }
    for (int k = 0; k < n1; ++k)
        if (!(h_tgt[k] >= 0.0)) return 1;
    if (n_active == 0) return 1;
    HostIO io{h_src, h_tgt, {f_src, f_src + n0, nullptr, nullptr}, {out, out + n1, nullptr, nullptr}};
    if (nf == 1) po::rc::remap_column_stream<1>(io, n0, n1, scheme, n_active, last);
    else po::rc::remap_column_stream<2>(io, n0, n1, scheme, n_active, last);
    return 0;
}

// The array formulation (used on the device for columns the sweep does not take), one field.
int remap_general_column(const double* h_src, const double* f_src, int n0, const double* h_tgt, int n1, int scheme,
                         double* out)
{
    if (n0 > 128 || n1 > 128) return 1;
    HostIO io{h_src, h_tgt, {f_src, nullptr, nullptr, nullptr}, {out, nullptr, nullptr, nullptr}};
    po::rc::remap_column_general<128>(io, 0, n0, n1, scheme);
    return 0;
}

}  // extern "C"
