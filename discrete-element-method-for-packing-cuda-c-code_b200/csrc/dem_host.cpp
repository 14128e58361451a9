// dem_host.cpp -- host side of the library: error strings, the hopp3d.inp
// deck and its reduced units, and the reference's output files (the initial
// states and material helpers are in dem_gen.cpp).
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
