// dem_host.cpp -- host side of the library: error strings, the hopp3d.inp
// deck and its reduced units, reproducible initial states, and the
// reference's output files.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#include <cuda_runtime.h>
#include "dem_b200.h"

namespace dem {

static thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
    const char* base = strrchr(file, '/');
    return fail(DEM_ERR_CUDA, "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), base ? base + 1 : file, line);
}

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

const char* dem_last_error_string(void) { return dem::g_err.c_str(); }

const char* dem_version(void) {
    return "dem_b200 1.0 (sm_100a; reference-compatible FP64 entry points; context API FP64 + mixed FP32/FP64)";
}

// ------------------------------------------------------------------- deck
int dem_read_deck(const char* path, dem_deck* d) {
    if (!path || !d) return fail(DEM_ERR_ARG, "dem_read_deck: null argument");
    memset(d, 0, sizeof(*d));
    FILE* f = fopen(path, "rb");
    if (!f) return fail(DEM_ERR_IO, "Cannot open file %s", path);
    // positional reads in the order of dempacking.cu:112-125
    int ok = 1;
    ok &= fscanf(f, "%d", &d->iforcemode) == 1;
    ok &= fscanf(f, "%lf %lf %lf", &d->emod, &d->vpois, &d->denp) == 3;
    ok &= fscanf(f, "%lf", &d->diam) == 1;
    ok &= fscanf(f, "%d", &d->ntot) == 1;
    ok &= fscanf(f, " %lf %u", &d->dt, &d->tstop) == 2;
    ok &= fscanf(f, " %lf %lf %lf", &d->dmt1, &d->dmt2, &d->thick) == 3;
    ok &= fscanf(f, " %lf %lf", &d->zht1, &d->zht2) == 2;
    ok &= fscanf(f, " %lf %d", &d->vel0, &d->nrings) == 2;
    ok &= fscanf(f, " %lf %lf", &d->ufricp, &d->ufricw) == 2;
    ok &= fscanf(f, " %lf %lf %lf %lf %lf", &d->dampnp, &d->damptp, &d->dampnw, &d->damptw, &d->cdamp) == 5;
    ok &= fscanf(f, " %lf %lf %lf", &d->stiffness, &d->dampcoeffn, &d->dampcoefft) == 3;
    ok &= fscanf(f, " %lf %lf", &d->upp, &d->upw) == 2;
    fclose(f);
    if (!ok) return fail(DEM_ERR_IO, "%s: malformed deck (expected the 12 numeric lines of hopp3d.inp)", path);
    if (!(d->diam > 0.0) || !(d->denp > 0.0) || !(d->emod > 0.0) || d->ntot <= 0 || !(d->dt > 0.0) ||
        !(d->dmt2 > 0.0) || !(d->thick > 0.0) || !(d->vpois < 1.0))
        return fail(DEM_ERR_IO, "%s: deck values out of range", path);
    // reduced units, dempacking.cu:141-149 (constants kept as written there)
    const double emod = 6.0 * d->emod / (3.14159265 * d->denp * 9.81 * d->diam);
    const double emodw = emod;
    const double nu = d->vpois;
    d->emod_red = emod;
    d->estarp = 1.33333333 * emod / (2.0 * (1.0 - nu * nu));
    d->estarw = 1.33333333 / ((1.0 - nu * nu) / emod + (1.0 - nu * nu) / emodw);
    // geometry, dempacking.cu:213-225,337-339
    d->world[0] = d->dmt2 / d->diam;
    d->world[1] = d->thick / d->diam;
    d->world[2] = d->zht1 / d->diam + d->zht2 / d->diam;
    d->upp_red = d->upp / d->diam;
    d->upw_red = d->upw / d->diam;
    return DEM_OK;
}

int dem_deck_material(const dem_deck* d, dem_material* m) {
    if (!d || !m) return fail(DEM_ERR_ARG, "dem_deck_material: null argument");
    m->pp = dem_contact{d->estarp, d->ufricp, d->vpois, d->dampnp, d->damptp, d->upp_red, 0.0};
    m->pw = dem_contact{d->estarw, d->ufricw, d->vpois, d->dampnw, d->damptw, d->upw_red, 0.0};
    return DEM_OK;
}

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

// ------------------------------------------------------------ output files
int dem_write_view(const char* path, const dem_deck* d) {
    if (!path || !d) return fail(DEM_ERR_ARG, "dem_write_view: null argument");
    FILE* f = fopen(path, "wb+");
    if (!f) return fail(DEM_ERR_IO, "Cannot open file %s", path);
    // dempacking.cu:231-234 (widths as written there; dmt1/dmt2 and the bed
    // heights in reduced units)
    fprintf(f, "number of particles=%4d\n", d->ntot);
    fprintf(f, "diameters =%6.3f\n", d->diam);
    fprintf(f, "time step=%f bed width=%6.3f thickniss=%6.3f\n", d->dt, d->dmt1 / d->diam, d->dmt2 / d->diam);
    fprintf(f, "glabal damping=%10.4f bed hbot=%10.4f htop=%10.4f\n", d->cdamp, d->zht1 / d->diam,
            d->zht1 / d->diam + d->zht2 / d->diam);
    fclose(f);
    return DEM_OK;
}

// ppor.dat line of dempacking.cu:774: it, N, contacts (pcntot/2), porosity,
// packing fraction, mean CN, max height.
int dem_write_ppor(const char* path, long long it, long long n, long long pcntot, double porosity, double packing,
                   double avercn, double maxhz) {
    FILE* f = fopen(path, "ab+");
    if (!f) return fail(DEM_ERR_IO, "Cannot open file %s", path);
    fprintf(f, "%8d %8d %8d %15.6f %15.6f %15.6f %15.6f\n", (int)it, (int)n, (int)(pcntot / 2), porosity, packing,
            avercn, maxhz);
    fclose(f);
    return DEM_OK;
}

// particle.dat zone of dempacking.cu:785-791 (metres: reduced * diam).
int dem_write_particles(const char* path, int zone, long long n, const double* pos, const double* rad, double diam) {
    if (!pos || !rad) return fail(DEM_ERR_ARG, "dem_write_particles: null argument");
    FILE* f = fopen(path, "ab+");
    if (!f) return fail(DEM_ERR_IO, "Cannot open file %s", path);
    fprintf(f, "ZONE T=\"ZONE%03d\"\n", zone);
    for (long long i = 0; i < n; i++)
        fprintf(f, "%15.6g%15.6g%15.6g%15.6g%8d\n", pos[3 * i] * diam, pos[3 * i + 1] * diam, pos[3 * i + 2] * diam,
                rad[i] * diam, (int)i);
    fclose(f);
    return DEM_OK;
}

// preflow.dat of dempacking.cu:812-820.
int dem_write_preflow(const char* path, long long it, long long n, long long itime, const double* pos,
                      const double* pdis, const double* angv) {
    if (!pos || !pdis || !angv) return fail(DEM_ERR_ARG, "dem_write_preflow: null argument");
    FILE* f = fopen(path, "wb+");
    if (!f) return fail(DEM_ERR_IO, "Cannot open file %s", path);
    fprintf(f, "%8d,%8d,%8d\n", (int)it, (int)n, (int)itime);
    for (long long i = 0; i < n; i++)
        fprintf(f, "%15.6f %15.6f %15.6f %15.6f %15.6f %15.6f %15.6f %15.6f %15.6f\n", pos[3 * i], pos[3 * i + 1],
                pos[3 * i + 2], pdis[3 * i], pdis[3 * i + 1], pdis[3 * i + 2], angv[3 * i], angv[3 * i + 1],
                angv[3 * i + 2]);
    fclose(f);
    return DEM_OK;
}

// preflow.dat reader: the format the writer above produces (the reference's
// own reader is commented out, dempacking.cu:361-367).  With pos == NULL only
// the header line is read (it, n, itime); otherwise n particles of 9 values
// (position, per-step displacement, per-step rotation) into arrays holding
// ncap particles.  The file keeps 6 decimals of each value.
int dem_read_preflow(const char* path, long long* it, long long* n, long long* itime, double* pos, double* pdis,
                     double* angv, long long ncap) {
    if (!path || !it || !n || !itime) return fail(DEM_ERR_ARG, "dem_read_preflow: null argument");
    FILE* f = fopen(path, "rb");
    if (!f) return fail(DEM_ERR_IO, "Cannot open file %s", path);
    long long a = 0, b = 0, c = 0;
    if (fscanf(f, " %lld , %lld , %lld", &a, &b, &c) != 3 || b < 0) {
        fclose(f);
        return fail(DEM_ERR_IO, "%s: malformed preflow header", path);
    }
    *it = a; *n = b; *itime = c;
    if (!pos) { fclose(f); return DEM_OK; }
    if (!pdis || !angv) { fclose(f); return fail(DEM_ERR_ARG, "dem_read_preflow: null array"); }
    if (b > ncap) { fclose(f); return fail(DEM_ERR_ARG, "dem_read_preflow: %lld particles exceed the arrays (%lld)", b, ncap); }
    for (long long i = 0; i < b; i++) {
        double v[9];
        if (fscanf(f, " %lf %lf %lf %lf %lf %lf %lf %lf %lf", v, v + 1, v + 2, v + 3, v + 4, v + 5, v + 6, v + 7,
                   v + 8) != 9) {
            fclose(f);
            return fail(DEM_ERR_IO, "%s: truncated at particle %lld", path, i);
        }
        for (int k = 0; k < 3; k++) { pos[3 * i + k] = v[k]; pdis[3 * i + k] = v[3 + k]; angv[3 * i + k] = v[6 + k]; }
    }
    fclose(f);
    return DEM_OK;
}

// timesteps.dat line of dempacking.cu:802.
int dem_write_timesteps(const char* path, double tret, long long it) {
    FILE* f = fopen(path, "ab+");
    if (!f) return fail(DEM_ERR_IO, "Cannot open file %s", path);
    fprintf(f, "%15.6f %15.6f\n", tret, (double)it);
    fclose(f);
    return DEM_OK;
}

// jobfinished and restart.dat of dempacking.cu:904-913.
int dem_write_finish(const char* jobfinished_path, const char* restart_path) {
    FILE* f = fopen(jobfinished_path, "wb");
    if (!f) return fail(DEM_ERR_IO, "Cannot open file %s", jobfinished_path);
    fprintf(f, "job finished\n");
    fclose(f);
    f = fopen(restart_path, "wb");
    if (!f) return fail(DEM_ERR_IO, "Cannot open file %s", restart_path);
    fprintf(f, "program comes to end!\n");
    fprintf(f, "%8d %8d\n", 1, 1);
    fclose(f);
    return DEM_OK;
}

}  // extern "C"
