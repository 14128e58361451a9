// dem_gen.cpp -- reproducible initial states and reduced-unit material
// helpers (host only, no CUDA).  Built into libdem_b200.so and, with
// -DDEM_GEN_STANDALONE, into the host-only libdem_gen.so, so that the GPU
// engine, the CPU oracle runs of the tests and the CPU timing of the
// reference step all start from the same bits without loading the GPU
// library.  The standalone build reports its errors through
// dem_gen_last_error().
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>
#include <algorithm>
#include "dem_b200.h"

namespace dem {
#ifdef DEM_GEN_STANDALONE
static thread_local std::string g_gen_err;
static int fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_gen_err = buf;
    return code;
}
#else
int fail(int code, const char* fmt, ...);
#endif

// SplitMix64 (Steele, Lea & Flood 2014): 64-bit state, one output per call.
struct SplitMix64 {
    unsigned long long s;
    explicit SplitMix64(unsigned long long seed) : s(seed) {}
    unsigned long long next() {
        unsigned long long z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }   // [0,1)
    double normal() {   // Box-Muller, one value per call
        double u1 = uniform(), u2 = uniform();
        if (u1 < 1e-300) u1 = 1e-300;
        return sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2);
    }
};
}  // namespace dem

using dem::fail;

extern "C" {

#ifdef DEM_GEN_STANDALONE
const char* dem_gen_last_error(void) { return dem::g_gen_err.c_str(); }
#endif

double dem_reduced_modulus(double E, double rho, double dref) { return 6.0 * E / (M_PI * rho * 9.81 * dref); }

double dem_estar(double E, double nu, double rho, double dref) {
    return (4.0 / 3.0) * dem_reduced_modulus(E, rho, dref) / (2.0 * (1.0 - nu * nu));
}

// Viscous normal damping for restitution e: beta = ln e / sqrt(ln^2 e + pi^2)
// and F = -2 sqrt(5/6) beta sqrt(S_n m*) v with S_n = 2 E* sqrt(R* delta);
// since sqrt(6 m* E* sqrt(R* delta)) = sqrt(3) sqrt(S_n m*), c = -2 sqrt(5/18) beta.
double dem_damp_from_restitution(double e) {
    if (!(e > 0.0) || e >= 1.0) return 0.0;
    const double le = log(e);
    const double beta = le / sqrt(le * le + M_PI * M_PI);
    return -2.0 * sqrt(5.0 / 18.0) * beta;
}

// ---------------------------------------------------------- initial states
int dem_gen_lattice(long long n, double a, int nx, int ny, double z0, double jit, double radius,
                    unsigned long long seed, double* pos, double* rad) {
    if (n <= 0 || nx <= 0 || ny <= 0 || !pos || !rad || !(a > 0.0)) return fail(DEM_ERR_ARG, "dem_gen_lattice: bad argument");
    dem::SplitMix64 rng(seed);
    const long long per = (long long)nx * ny;
    for (long long i = 0; i < n; i++) {
        const long long L = i / per, r = i % per;
        const int iy = (int)(r / nx), ix = (int)(r % nx);
        double x = (ix - 0.5 * (nx - 1)) * a;
        double y = (iy - 0.5 * (ny - 1)) * a;
        double z = z0 + (double)L * a;
        x += (2.0 * rng.uniform() - 1.0) * jit;
        y += (2.0 * rng.uniform() - 1.0) * jit;
        z += (2.0 * rng.uniform() - 1.0) * jit;
        pos[3 * i] = x; pos[3 * i + 1] = y; pos[3 * i + 2] = z;
        rad[i] = (double)(float)radius;
    }
    return DEM_OK;
}

// Radii are returned as FP32-representable doubles, so a mixed-precision run
// stores them without rounding.
int dem_gen_radii(long long n, int kind, double a, double b, double c, double d, unsigned long long seed, double* rad) {
    if (n <= 0 || !rad) return fail(DEM_ERR_ARG, "dem_gen_radii: bad argument");
    dem::SplitMix64 rng(seed);
    if (kind == DEM_RADII_MONO) {
        for (long long i = 0; i < n; i++) rad[i] = (double)(float)a;
    } else if (kind == DEM_RADII_LOGNORMAL) {
        if (!(a > 0.0) || !(c < d) || !(c > 0.0)) return fail(DEM_ERR_ARG, "dem_gen_radii: bad lognormal range");
        const double la = log(a);
        for (long long i = 0; i < n; i++) {
            double r;
            int tries = 0;
            do {
                r = exp(la + b * rng.normal());
                if (++tries > 1000000) return fail(DEM_ERR_ARG, "dem_gen_radii: truncation range never hit");
            } while (r < c || r > d);
            rad[i] = (double)(float)r;
        }
    } else if (kind == DEM_RADII_BIDISPERSE) {
        for (long long i = 0; i < n; i++) rad[i] = (double)(float)(i < n / 2 ? a : b);
        for (long long i = n - 1; i > 0; i--) {   // Fisher-Yates
            long long j = (long long)(rng.uniform() * (double)(i + 1));
            if (j > i) j = i;
            std::swap(rad[i], rad[j]);
        }
    } else {
        return fail(DEM_ERR_ARG, "dem_gen_radii: unknown kind %d", kind);
    }
    return DEM_OK;
}

// Random sequential addition in the open box (-Wx/2..Wx/2, -Wy/2..Wy/2,
// 0..Wz) with wall clearance r and no overlaps; a cell grid of edge 2 r_max
// finds the placed neighbours.
int dem_gen_rsa(long long n, const double world[3], const double* rad, unsigned long long seed, double* pos) {
    if (n <= 0 || !world || !rad || !pos) return fail(DEM_ERR_ARG, "dem_gen_rsa: bad argument");
    double rmax = 0.0;
    for (long long i = 0; i < n; i++) rmax = std::max(rmax, rad[i]);
    const double cs = 2.0 * rmax;
    const long long gx = std::max(1LL, (long long)(world[0] / cs)), gy = std::max(1LL, (long long)(world[1] / cs)),
                    gz = std::max(1LL, (long long)(world[2] / cs));
    const double ex = world[0] / gx, ey = world[1] / gy, ez = world[2] / gz;   // cell edges >= cs
    std::vector<long long> head((size_t)(gx * gy * gz), -1), next((size_t)n, -1);
    dem::SplitMix64 rng(seed);
    const double hx = 0.5 * world[0], hy = 0.5 * world[1];
    for (long long i = 0; i < n; i++) {
        const double r = rad[i];
        if (2.0 * r >= world[0] || 2.0 * r >= world[1] || 2.0 * r >= world[2])
            return fail(DEM_ERR_ARG, "dem_gen_rsa: particle does not fit the box");
        bool placed = false;
        for (int attempt = 0; attempt < 100000 && !placed; attempt++) {
            const double x = -hx + r + rng.uniform() * (world[0] - 2.0 * r);
            const double y = -hy + r + rng.uniform() * (world[1] - 2.0 * r);
            const double z = r + rng.uniform() * (world[2] - 2.0 * r);
            const long long cx = std::min(gx - 1, (long long)((x + hx) / ex));
            const long long cy = std::min(gy - 1, (long long)((y + hy) / ey));
            const long long cz = std::min(gz - 1, (long long)(z / ez));
            bool ok = true;
            for (long long zz = std::max(0LL, cz - 1); ok && zz <= std::min(gz - 1, cz + 1); zz++)
                for (long long yy = std::max(0LL, cy - 1); ok && yy <= std::min(gy - 1, cy + 1); yy++)
                    for (long long xx = std::max(0LL, cx - 1); ok && xx <= std::min(gx - 1, cx + 1); xx++)
                        for (long long j = head[(size_t)((zz * gy + yy) * gx + xx)]; j >= 0; j = next[(size_t)j]) {
                            const double dx = pos[3 * j] - x, dy = pos[3 * j + 1] - y, dz = pos[3 * j + 2] - z;
                            const double s = r + rad[j];
                            if (dx * dx + dy * dy + dz * dz < s * s) { ok = false; break; }
                        }
            if (!ok) continue;
            pos[3 * i] = x; pos[3 * i + 1] = y; pos[3 * i + 2] = z;
            const size_t c = (size_t)((cz * gy + cy) * gx + cx);
            next[(size_t)i] = head[c];
            head[c] = i;
            placed = true;
        }
        if (!placed) return fail(DEM_ERR_ARG, "dem_gen_rsa: could not place particle %lld (box too full)", i);
    }
    return DEM_OK;
}

}  // extern "C"
