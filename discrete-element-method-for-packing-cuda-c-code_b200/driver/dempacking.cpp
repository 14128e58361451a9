// dempacking -- deck-compatible driver of the B200 DEM step (the role of the
// reference's main loop, dempacking.cu:28-918), on the context API.
//
//   dempacking [deck=hopp3d.inp] [--precision mixed|fp64] [--relist K]
//              [--seed S] [--steps N] [--stacked]
//
// Reads the hopp3d.inp deck (dempacking.cu:107-126), converts to reduced
// units (:141-149,213-225) and pours the packing as the reference does
// (:242-316, :373-534): ntot spheres of diameter 1 with injection states on
// the deck's injection lattice (nrings x nringsy sites, spacing dmt2/nrings by
// thick/nringsy) at height hopzt - 5, the deck's speed vel0 in a random
// downward direction (:302-309, seeded instead of rand()), joining the
// system a layer of nplayer at a time every tnewpar = 0.5 time units
// (dem_set_pour).  --stacked places all ntot at once in layers stacked from
// the floor instead.  Runs tstop steps and writes the reference's files:
// view.dat, ppor.dat every 1000 steps, particle.dat at step 1 and every
// 50,000 steps, timesteps.dat every 1000 steps, preflow.dat when the run
// passes 3600 s of CPU time (then every 7200 s), jobfinished and restart.dat
// at the end; particle counts are those in the system.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>
#include "dem_b200.h"

static int die(int rc, const char* what) {
    fprintf(stderr, "dempacking: %s failed (%d): %s\n", what, rc, dem_last_error_string());
    return 1;
}

int main(int argc, char** argv) {
    const char* deck_path = "hopp3d.inp";
    int precision = DEM_PREC_MIXED, relist = 20, stacked = 0;
    unsigned long long seed = 20261203ull;
    long long steps_override = -1;
    for (int a = 1; a < argc; a++) {
        if (!strcmp(argv[a], "--precision") && a + 1 < argc) {
            precision = strcmp(argv[++a], "fp64") ? DEM_PREC_MIXED : DEM_PREC_FP64;
        } else if (!strcmp(argv[a], "--relist") && a + 1 < argc) {
            relist = atoi(argv[++a]);
        } else if (!strcmp(argv[a], "--seed") && a + 1 < argc) {
            seed = strtoull(argv[++a], nullptr, 10);
        } else if (!strcmp(argv[a], "--steps") && a + 1 < argc) {
            steps_override = atoll(argv[++a]);
        } else if (!strcmp(argv[a], "--stacked")) {
            stacked = 1;
        } else {
            deck_path = argv[a];
        }
    }
    dem_deck d;
    int rc = dem_read_deck(deck_path, &d);
    if (rc) return die(rc, "dem_read_deck");
    // deck echo (dempacking.cu:128-139)
    printf("%d\n%lf %lf %lf\n%lf\n%d\n%lf %u\n%lf %lf %lf\n%lf %lf\n%lf %d\n%lf %lf\n%lf %lf %lf %lf %lf\n"
           "%lf %lf %lf\n%lf %lf\n",
           d.iforcemode, d.emod, d.vpois, d.denp, d.diam, d.ntot, d.dt, d.tstop, d.dmt1, d.dmt2, d.thick, d.zht1,
           d.zht2, d.vel0, d.nrings, d.ufricp, d.ufricw, d.dampnp, d.damptp, d.dampnw, d.damptw, d.cdamp,
           d.stiffness, d.dampcoeffn, d.dampcoefft, d.upp, d.upw);
    if ((rc = dem_write_view("view.dat", &d))) return die(rc, "view.dat");
    const long long n = d.ntot;
    const double W = d.world[0], T = d.world[1];
    // injection sites (dempacking.cu:243-282): nrings x nringsy, or one site
    // when the box is narrower than about four diameters
    int nx = (int)W - 3, ny = (int)T - 3;
    if (!(0.5 * W > 1.99) || nx < 1 || ny < 1) nx = ny = 1;
    const long long nplayer = (long long)nx * ny;
    const double ax = W / nx, ay = T / ny;
    const double az = 1.05;
    const double hopzt = d.world[2], zp0 = hopzt - 5.0;
    if (!stacked && !(zp0 > 0.5)) { fprintf(stderr, "dempacking: hopper shorter than the injection height\n"); return 1; }
    std::vector<double> pos(3 * n), pdis(3 * n, 0.0), rad(n, 0.5);
    unsigned long long s = seed;
    auto urand = [&]() {   // SplitMix64
        unsigned long long z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    };
    const double pi = 4.0 * atan(1.0);
    for (long long i = 0; i < n; i++) {
        const long long layer = i / nplayer, site = i % nplayer;
        const int ix = (int)(site / ny), iy = (int)(site % ny);
        pos[3 * i] = nx > 1 ? (ix + 0.5) * ax - 0.5 * W : 0.0;
        pos[3 * i + 1] = ny > 1 ? (iy + 0.5) * ay - 0.5 * T : 0.0;
        pos[3 * i + 2] = stacked ? 0.5 + 0.05 + layer * az : zp0;
        double ang = pi * (urand() * .33333 + .33333);
        pdis[3 * i + 2] = -d.vel0 * sin(ang) * d.dt;
        double dxy = -d.vel0 * cos(ang) * d.dt;
        ang = 2.0 * pi * urand();
        pdis[3 * i] = dxy * cos(ang);
        pdis[3 * i + 1] = dxy * sin(ang);
    }
    double world[3] = {W, T, stacked ? std::max(d.world[2], pos[3 * (n - 1) + 2] + 2.0) : hopzt};
    dem_config cfg;
    memset(&cfg, 0, sizeof(cfg));
    cfg.n = n;
    cfg.precision = precision;
    cfg.relist_interval = relist;
    for (int a = 0; a < 3; a++) cfg.world[a] = world[a];
    cfg.dt = d.dt;
    cfg.skin = 0.55;        // cub - cua of the reference (neiglist.cu:27-28)
    cfg.cell = 1.55;        // dempacking.cu:329-331
    cfg.density = 1.0;
    dem_ctx* ctx = nullptr;
    if ((rc = dem_create(&cfg, &ctx))) return die(rc, "dem_create");
    dem_material mat;
    dem_deck_material(&d, &mat);
    if ((rc = dem_set_material(ctx, &mat))) return die(rc, "dem_set_material");
    if ((rc = dem_upload_state(ctx, pos.data(), pdis.data(), nullptr, rad.data()))) return die(rc, "dem_upload_state");
    // poured packing: no particle in at first, a layer every 0.5 time units
    // (tnewpar, dempacking.cu:380)
    if (!stacked && (rc = dem_set_pour(ctx, nplayer, 0.5, 0))) return die(rc, "dem_set_pour");
    const long long tstop = steps_override >= 0 ? steps_override : (long long)d.tstop;
    const clock_t start = clock();
    double realtime = 3600.0;
    int nparticledat = 0;
    std::vector<double> hp(3 * n), hd(3 * n), ha(3 * n);
    long long it = 0;
    while (it < tstop) {
        // advance to the next output point in one call (graph windows inside)
        long long next = it + 1;
        if (it >= 1) {
            long long to1000 = ((it / 1000) + 1) * 1000;
            long long to50k = ((it / 50000) + 1) * 50000;
            next = std::min(std::min(to1000, to50k), tstop);
        }
        if ((rc = dem_step_n(ctx, next - it))) return die(rc, "dem_step_n");
        it = next;
        dem_scalars sc;
        rc = dem_get_scalars(ctx, &sc);
        if (rc) return die(rc, "dem_get_scalars");
        if (sc.status != DEM_OK) return die(sc.status, "the step");
        long long na = n;   // particles in the system (m_numParticles)
        if ((rc = dem_active_count(ctx, &na))) return die(rc, "dem_active_count");
        if (it % 1000 == 0) {
            const double pcntot = 2.0 * (double)sc.contacts;
            const double avercn = pcntot / (na * 1.0 + 1.0e-30);
            const double packing = sc.packing_fraction;
            if ((rc = dem_write_ppor("ppor.dat", it, na, (long long)pcntot, 1.0 - packing, packing, avercn,
                                     sc.maxhz)))
                return die(rc, "ppor.dat");
            printf("%8d %8d %8d %15.6f %15.6f %15.6f %15.6f\n", (int)it, (int)na, (int)(pcntot / 2), 1.0 - packing,
                   packing, avercn, sc.maxhz);
        }
        if (it % 50000 == 0 || it == 1) {
            if ((rc = dem_download_state(ctx, hp.data(), hd.data(), ha.data()))) return die(rc, "download");
            nparticledat++;
            if ((rc = dem_write_particles("particle.dat", nparticledat, na, hp.data(), rad.data(), d.diam)))
                return die(rc, "particle.dat");
        }
        const double tret = (double)(clock() - start) / CLOCKS_PER_SEC;
        if (it % 1000 == 0) dem_write_timesteps("timesteps.dat", tret, it);
        if (tret >= realtime) {
            if ((rc = dem_download_state(ctx, hp.data(), hd.data(), ha.data()))) return die(rc, "download");
            long long na = n;
            if ((rc = dem_active_count(ctx, &na))) return die(rc, "dem_active_count");
            dem_write_preflow("preflow.dat", it, na, 0, hp.data(), hd.data(), ha.data());
            realtime += 7200.0;
        }
    }
    dem_destroy(ctx);
    if ((rc = dem_write_finish("jobfinished", "restart.dat"))) return die(rc, "finish files");
    printf("program comes to end!\n");
    return 0;
}
