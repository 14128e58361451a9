/*
 * dem_b200.h -- C ABI of the B200 (sm_100a) DEM packing time step.
 *
 * Two layers are exported from libdem_b200.so:
 *
 *  1. Reference-compatible entry points.  They keep the names, argument order
 *     and argument meaning of the host launch wrappers in the reference's
 *     extern "C" block (particleSystem.cu:13-424) plus the SDK RadixSort call
 *     (dempacking.cu:553-555), so dempacking.cu's step loop can link against
 *     this library instead.  All array arguments are DEVICE pointers in the
 *     reference's layout (xyz-interleaved double, i.e. double3 AoS).  The one
 *     change: every call returns an int status (DEM_OK ...) instead of calling
 *     exit() (particleSystem.cu:15-23); a caller that ignores the return value
 *     behaves as before.  The __constant__ symbols Par/ParW/cua/cub that the
 *     reference fills with cudaMemcpyToSymbol (dempacking.cu:355-356,
 *     neiglist.cu:27-49) are set through setMaterialProperties/setListCutoff.
 *
 *  2. The context API (dem_*).  An opaque dem_ctx owns structure-of-arrays
 *     device buffers, a CSR contact-candidate list and CUDA graphs of whole
 *     re-list windows; dem_step_n advances the packing with no host sync.
 *     Precision is FP64 throughout (DEM_PREC_FP64) or mixed (DEM_PREC_MIXED:
 *     FP32 hashing/list/forces/accumulation, FP64 positions, velocities and
 *     tangential history).
 *
 * Units are the reference's reduced units (dempacking.cu:146-149,213-225):
 * length = particle diameter d, mass = rho*pi*d^3/6, force = that mass times
 * g, time = sqrt(d/g).  pdis and angv are per-step displacement and rotation
 * (velocity*dt, angular velocity*dt), as in the reference.
 */
#ifndef DEM_B200_H
#define DEM_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status -- */
#define DEM_OK              0
#define DEM_ERR_ARG         1  /* bad argument (null pointer, size, mode)          */
#define DEM_ERR_CUDA        2  /* a CUDA runtime call or kernel launch failed      */
#define DEM_ERR_CAPACITY    3  /* neighbour / pair capacity exceeded (list cut)    */
#define DEM_ERR_NONFINITE   4  /* NaN or Inf appeared in positions/velocities      */
#define DEM_ERR_SKIN        5  /* a particle moved more than skin/2 inside a window */
#define DEM_ERR_IO          6  /* deck / output file error                          */
#define DEM_ERR_STATE       7  /* call out of order (e.g. step before upload)       */
#define DEM_ERR_TIMEOUT     8  /* a bounded device-side wait ran out (window kernel's grid barrier, re-list scans) */

/* Text of the last error raised on the calling host thread. */
const char* dem_last_error_string(void);
/* Library build identification (arch, precision modes). */
const char* dem_version(void);

/* ============================================================================
 * 1. Reference-compatible entry points (device pointers, reference layout)
 * ==========================================================================*/

/* Key/value record of the SDK radix sort used at dempacking.cu:553-555. */
typedef struct {
    unsigned int key;
    unsigned int value;
} KeyValuePair;

/* Material constants, same fields and order as the reference's __constant__
 * structs (neiglist.cu:32-47).  estar* already contain the 4/3 Hertz factor
 * (dempacking.cu:148-149); upp/upw are rolling-friction lengths in units of d. */
typedef struct {
    double estarp, ufricp, vpois, dampnp, damptp, upp;
} Matproperties;
typedef struct {
    double estarw, ufricw, vpoisw, dampnw, damptw, upw;
} Wallproperties;

/* Replaces cudaMemcpyToSymbol(Par/ParW, ...) at dempacking.cu:355-356. */
int setMaterialProperties(const Matproperties* par, const Wallproperties* parw);
/* Replaces the __constant__ cua/cub of neiglist.cu:27-28: contact distance
 * (cua) and candidate cut-off distance (cub) between centres, in units of d.
 * neighborarray lists j when |x_i - x_j| < cub; updateposition raises the
 * re-list flag when |q_i| > 0.5*(cub-cua) (neiglist.cu:335,370). */
int setListCutoff(double cua, double cub);
/* Stream used by all reference-compatible calls (default: legacy stream 0). */
int dem_compat_set_stream(void* cuda_stream);

/* RadixSort(pData0, pData1, elements, keybits)  -- dempacking.cu:553-555.
 * Stable LSD sort of `elements` records by the low `keybits` bits of key;
 * result in pData0, pData1 is the ping-pong buffer.  Scratch for the digit
 * histograms is allocated by the library on the first call per device and
 * kept until exit. */
int RadixSort(KeyValuePair* pData0, KeyValuePair* pData1,
              unsigned int elements, unsigned int keybits);

/* RadixSortNoAlloc(pData0, pData1, elements, keybits) -- no counterpart in the
 * reference.  RadixSort for callers that cannot allocate device memory (a
 * host loop whose own pool allocator owns the GPU's memory, or a
 * latency-critical loop that must not pay a first-call allocation): the same
 * stable sort and result, with its scratch in a fixed device array inside the
 * library instead of cudaMalloc'd memory.  At most 4,194,304 records (larger
 * requests return DEM_ERR_ARG); the array (about 2 MiB) is held on every GPU
 * that loads the library until exit.  The first call on each device sets up
 * the array's address, which may also load the library's device code (and
 * with it reserve device memory) under CUDA's lazy module loading: make that
 * first call during set-up, before any stream capture; later calls allocate
 * nothing.  All calls share the array: calls that overlap on the GPU race and
 * must be serialised. */
int RadixSortNoAlloc(KeyValuePair* pData0, KeyValuePair* pData1,
                     unsigned int elements, unsigned int keybits);

/* calcHash  -- particleSystem.cu:27-45, kernel neiglist.cu:54-97.
 * particleHash[2i] = clamped linear cell id of particle i, [2i+1] = i. */
int calcHash(double* Pos, unsigned int* particleHash, unsigned int gridSize[3],
             double cellSize[3], double worldOrigin[3], int numBodies);

/* findCellStart  -- particleSystem.cu:49-64, kernel neiglist.cu:102-120.
 * cellStart[c] = first sorted index with key c, 0xffffffff if empty. */
int findCellStart(unsigned int* particleHash, unsigned int* cellStart,
                  int numBodies, unsigned int numGridCells);

/* neighborarray  -- particleSystem.cu:67-97 (kernel neighborarrayD absent from
 * the reference).  Row i of Anei (maxParticlesPerCell slots) holds the
 * njgi[i] neighbours j>i in ascending id order, then the njli[i] neighbours
 * j<i in ascending order; unused slots are 0xffffffff (particleSystem.cu:83).
 * Returns DEM_ERR_CAPACITY if a row would overflow (the row is cut). */
int neighborarray(double* pos, unsigned int* particleHash, unsigned int* cellStart,
                  unsigned int gridSize[3], double cellSize[3], double worldOrigin[3],
                  int maxParticlesPerCell, int numBodies,
                  unsigned int* Anei, unsigned int* njgi, unsigned int* njli);

/* prefixsum  -- particleSystem.cu:126-140.  oldsjgi <- sjgi; sjgi = inclusive
 * scan of njgi; *totalcontacts (HOST) = sjgi[numBodies-1].  Synchronises. */
int prefixsum(unsigned int numBodies, unsigned int* njgi, unsigned int* sjgi,
              unsigned int* oldsjgi, unsigned int* totalcontacts);

/* pairlist  -- particleSystem.cu:143-191 (kernel pairlistD absent).
 * Pairs of i occupy [sjgi[i]-njgi[i], sjgi[i]): Lp=i, Ln=j (j>i ascending).
 * Aref row i: list slot of each neighbour in Anei row order.  Tangential
 * history dispt (double3) / fricp of pair (i,j) is copied from the previous
 * list (olddispt/oldfricp at the slot where oldLn==j inside i's previous range
 * [oldsjgi[i-1], oldsjgi[i])), else zero. */
int pairlist(unsigned int* sjgi, unsigned int* oldsjgi, unsigned int* oldLn,
             unsigned int* Anei, unsigned int* njgi, unsigned int* njli,
             double* olddispt, double* oldfricp,
             int maxParticlesPerCell, int maxCnPerParticle, unsigned int numBodies,
             unsigned int* Aref, unsigned int* Lp, unsigned int* Ln,
             double* dispt, double* fricp);

/* calculateforcepair  -- particleSystem.cu:194-240, kernel neiglist.cu:156-233.
 * One thread per candidate pair: Hertz-Mindlin normal + damping, Mindlin
 * tangential spring with Coulomb cap, rolling resistance.  forcepair = force
 * on Lp (the Ln side receives minus it), torqpairi/j = torques on Lp/Ln,
 * contactpair = 1 when touching.  dispt/fricp and olddispt/oldfricp/oldLn are
 * updated as at neiglist.cu:211-231. */
int calculateforcepair(double* pos, double* pdis, double* angv, double* rad, double* rmass,
                       unsigned int* Lp, unsigned int* Ln, unsigned int* oldLn,
                       double* dispt, double* fricp, double* olddispt, double* oldfricp,
                       double dt,
                       double* forcepair, double* torqpairi, double* torqpairj,
                       unsigned int* contactpair, unsigned int totalcontacts);

/* sumallforcei  -- particleSystem.cu:243-277 (kernel sumallforceiD absent).
 * Gather through Aref: forcei = sum own-pair forces - sum forces of pairs
 * where i is Ln; torquei likewise with torqpairi / torqpairj; contacti =
 * number of touching pairs.  Deterministic, no atomics. */
int sumallforcei(int maxParticlesPerCell, int numBodies, unsigned int* njgi, unsigned int* njli,
                 double* forcepair, double* torqpairi, double* torqpairj,
                 unsigned int* contactpair, unsigned int* Aref,
                 double* forcei, double* torquei, unsigned int* contacti);

/* calculateforceiw  -- particleSystem.cu:279-313, kernel neiglist.cu:238-306.
 * Adds gravity (0,0,-m) and flat-wall contact (x=+-Wx/2, y=+-Wy/2, z=0, open
 * top) to forcei/torquei (pair sums are used only if totalcontacts != 0).
 * One wall-history slot per particle (disptw/fricpw). */
int calculateforceiw(double worldSize[3], double* pos, double* pdis, double* angv,
                     double* rad, double* rmass, double dt, unsigned int totalcontacts,
                     int numBodies, double* disptw, double* fricpw,
                     double* forcei, double* torquei);

/* updateposition  -- particleSystem.cu:315-384, kernel neiglist.cu:308-409.
 * Symplectic Euler in displacement form; *iall (HOST) = 1 if any |q_i| >
 * 0.5*(cub-cua), *maxhz (HOST) = max(0, max_i z_i).  Synchronises. */
int updateposition(double worldSize[3], int numBodies, double* pos, double* pdis,
                   double* angv, double* rmass, double* inert, double* forcei,
                   double* torquei, double* qi, double dt, double cdamp,
                   unsigned int* iall, double* maxhz);

/* outputporositycn  -- particleSystem.cu:386-422.  *pcntot (HOST) = sum of
 * contacti.  Synchronises. */
int outputporositycn(unsigned int numBodies, unsigned int* contacti, double maxhz,
                     double worldSize[3], unsigned int* pcntot);

/* ============================================================================
 * 2. Context API (structure-of-arrays engine, CUDA-graph windows)
 * ==========================================================================*/
#define DEM_PREC_FP64   0
#define DEM_PREC_MIXED  1

/* Force decomposition.  PCCP (the reference's, README.md:4-6): one thread per
 * candidate pair writes pair forces, one thread per particle gathers them.
 * PP (the paper's particle-parallel form, Figure 1(b)): one thread per
 * particle evaluates all of its pairs (each pair twice, bit-identically) and
 * integrates, one kernel per step, with ping-pong state buffers. */
#define DEM_FORCE_PCCP  0
#define DEM_FORCE_PP    1

typedef struct dem_ctx dem_ctx;

/* Contact parameters in reduced units.  Rolling-friction length of a pair is
 * roll + roll_rel * R*, with R* = r_i r_j/(r_i+r_j) (R* = r for a wall). */
typedef struct {
    double estar;    /* (4/3) E/(2(1-nu^2)) reduced, as dempacking.cu:148      */
    double mu;       /* sliding friction                                       */
    double nu;       /* Poisson ratio (slip length mu(2-nu)/(2(1-nu)) delta)   */
    double damp_n;   /* normal damping coefficient (hopp3d.inp line 10)        */
    double damp_t;   /* tangential damping coefficient                         */
    double roll;     /* rolling-friction length, units of d                    */
    double roll_rel; /* rolling-friction length per unit R*                    */
} dem_contact;

typedef struct {
    dem_contact pp;  /* particle-particle */
    dem_contact pw;  /* particle-wall     */
} dem_material;

typedef struct {
    long long n;            /* particles                                        */
    int precision;          /* DEM_PREC_FP64 / DEM_PREC_MIXED                   */
    int relist_interval;    /* steps per window (re-list at window start)       */
    double world[3];        /* box Wx, Wy, Wz; origin (-Wx/2,-Wy/2,0)           */
    double dt;              /* reduced time step                                */
    double skin;            /* list skin: candidates |dx| < r_i+r_j+skin        */
    double cell;            /* cell edge; 0 -> 2*r_max+skin (+1e-4)             */
    double density;         /* mass = density*8r^3 (1 in reduced units)         */
    long long pair_capacity;/* half-list capacity; 0 -> 8*n                     */
    int force_mode;         /* DEM_FORCE_PCCP (default 0) / DEM_FORCE_PP        */
} dem_config;

/* Per-step observables (reference ppor.dat columns, dempacking.cu:766-776). */
typedef struct {
    long long step;          /* steps taken since upload                        */
    long long pairs;         /* candidate pairs in the current list (half list) */
    long long contacts;      /* touching pairs (= pcntot/2)                     */
    double maxhz;            /* max(0, max_i z_i)                               */
    double packing_fraction; /* sum (4/3)pi r^3 / (Wx*Wy*maxhz)                 */
    double mean_cn;          /* 2*contacts/n                                    */
    long long relists;       /* list builds since upload                        */
    int status;              /* sticky device status (DEM_OK / DEM_ERR_*)       */
    int max_row;             /* largest per-particle candidate count seen       */
} dem_scalars;

int dem_create(const dem_config* cfg, dem_ctx** out);
int dem_destroy(dem_ctx* ctx);
int dem_set_stream(dem_ctx* ctx, void* cuda_stream);
int dem_set_material(dem_ctx* ctx, const dem_material* mat);
/* Host AoS (xyz-interleaved) double arrays of length 3n (rad: n).  pdis/angv
 * may be NULL (zero).  Resets histories and forces a re-list.  The context
 * stores the particles sorted by cell (locality of every gather and scatter;
 * the order is computed on the device and the call waits for it; 64
 * particles or fewer, or environment DEM_B200_REORDER=0, keep the caller's
 * order); every result -- states, forces, pairs, cells, radius gradients --
 * is returned in the caller's order and ids.  The _device form keeps the
 * caller's order. */
int dem_upload_state(dem_ctx* ctx, const double* pos, const double* pdis,
                     const double* angv, const double* rad);
/* Same with device pointers (AoS double), no host copy. */
int dem_upload_state_device(dem_ctx* ctx, const double* pos, const double* pdis,
                            const double* angv, const double* rad);
int dem_download_state(dem_ctx* ctx, double* pos, double* pdis, double* angv);
int dem_download_state_device(dem_ctx* ctx, double* pos, double* pdis, double* angv);
/* Advance nsteps (any count; whole windows replay a captured CUDA graph). */
int dem_step_n(dem_ctx* ctx, long long nsteps);
/* Synchronises; observables of the last step and the sticky status. */
int dem_get_scalars(dem_ctx* ctx, dem_scalars* out);
/* Observables without a host wait.  dem_scalars_enqueue queues, on the
 * context's stream, the device-to-host copy of what dem_get_scalars reads
 * (status, pair count, the last step's per-block partials) into `raw`, host
 * memory of dem_scalars_raw_bytes bytes (pinned memory makes the copy
 * asynchronous), and returns at once; once the stream has passed the copy
 * (dem_synchronize or any call that waits), dem_scalars_from_raw reduces it
 * to the dem_scalars of that moment, with dem_get_scalars' return codes.
 * Each enqueue needs its own buffer until it has been reduced. */
int dem_scalars_raw_bytes(dem_ctx* ctx, long long* bytes);
int dem_scalars_enqueue(dem_ctx* ctx, void* raw);
int dem_scalars_from_raw(dem_ctx* ctx, const void* raw, dem_scalars* out);
int dem_synchronize(dem_ctx* ctx);
/* Record per-particle force/torque/contact count of each step into device
 * buffers (off by default; costs 52 bytes per particle-step of writes). */
int dem_record_forces(dem_ctx* ctx, int on);
/* Per-particle force/torque/contact count of the last step (host, AoS);
 * needs dem_record_forces(ctx, 1) before the step. */
int dem_download_forces(dem_ctx* ctx, double* force, double* torque, unsigned int* contacts);
/* Current half list in canonical order (i ascending, then j): host arrays of
 * capacity `cap`; *npairs receives the count. */
int dem_download_pairs(dem_ctx* ctx, unsigned int* lp, unsigned int* ln,
                       double* hist, long long cap, long long* npairs);
/* Sorted (cell key, particle id) of the last re-list and cell ranges. */
int dem_download_cells(dem_ctx* ctx, unsigned int* keys, unsigned int* ids,
                       unsigned int* cell_start, unsigned int* cell_end, long long ncells_cap);
int dem_grid_info(dem_ctx* ctx, unsigned int grid[3], double* cell, long long* ncells);
/* Mean kernel time of the last dem_step_n call per kernel family (ms):
 * out[0]=re-list, out[1]=pair force, out[2]=particle update.  Enabled by
 * dem_set_profiling(ctx,1); adds events, so off for timing runs. */
int dem_set_profiling(dem_ctx* ctx, int on);
int dem_kernel_times(dem_ctx* ctx, double out[3]);
/* Event timing inside the window graphs: while on, whole windows replay a
 * second graph that also records CUDA events around the re-list and the step
 * kernels (plain windows carry no event nodes).  dem_window_kernel_times
 * gives the times (ms) of the last such window: out[0]=re-list; per-step
 * path: out[1]=pair force per step, out[2]=bound-particle update per step,
 * out[3]=the forked free-particle kernel (whole window); window-kernel path
 * (PCCP default): out[4]=the window kernel (all steps).  PP mode: out[1] ~ 0,
 * out[2] the fused step. */
/* Check of the window kernel's bounded grid-barrier wait (no fault, no
 * hang): on the context's stream, one block waits for a barrier arrival that
 * never comes; the wait gives up after about 1 s, records the timeout in the
 * status word (dem_get_scalars then reports DEM_ERR_TIMEOUT until the next
 * upload) and the launch ends.  DEM_OK when the timeout was reported;
 * *waited_ms receives the time the block waited.  At a re-list boundary
 * (DEM_ERR_STATE otherwise). */
int dem_check_barrier_timeout(dem_ctx* ctx, double* waited_ms);
int dem_set_window_timing(dem_ctx* ctx, int on);
int dem_window_kernel_times(dem_ctx* ctx, double out[5]);
/* Work of the current list's window (waits for the context's stream):
 * *bound = particles with a listed pair or a wall candidacy (stepped with the
 * pair phase), *wall_candidates = particles near a wall, *pairs = listed
 * pairs; the others step under gravity alone until the next re-list.
 * *batched = 1 when the bound particles' connected components (through the
 * pair list) were small enough to be stepped as cluster batches, one block
 * per batch in shared memory, 0 when the grid-barrier window kernel stepped
 * them (a dense bed is one large component), -1 when the context does not
 * batch (PP mode, DEM_B200_BATCH=0, per-step kernels).  Any pointer may be
 * NULL.  No
 * counterpart in the reference (it steps every particle the same way). */
int dem_window_work(dem_ctx* ctx, long long* bound, long long* wall_candidates, long long* pairs, int* batched);

/* Checkpoint / resume (the reference's restart reader is commented out,
 * dempacking.cu:361-367, and its preflow.dat has no contact history).
 * dem_save_state writes the whole engine state at a re-list boundary (step a
 * multiple of relist_interval, else DEM_ERR_STATE): particle state, radii,
 * displacement-since-list words, wall history, the previous pair list with
 * its FP64 tangential history, step counters, material and a pour in
 * progress (binary, native byte order, this library only).  dem_load_state
 * restores it into a context of the same n, precision, force mode and
 * relist_interval (DEM_ERR_ARG otherwise; DEM_ERR_IO for a file that is not
 * one, or whose pair list is malformed); stepping on gives the same states
 * bit for bit as the saved context would. */
int dem_save_state(dem_ctx* ctx, const char* path);
int dem_load_state(dem_ctx* ctx, const char* path);

/* Poured packing: the reference's layer injection (dempacking.cu:373-534),
 * replacing its download / free / malloc / upload of every array per layer
 * with buffers sized once for all particles.  The context's n particles are
 * the run's ntot; the state uploaded last (dem_upload_state*) holds their
 * injection states (position, displacement per step, rotation, radius).
 * After dem_set_pour only the first n_active are in the system.  Before each
 * step (reference step it = completed steps + 1, time = dt*it,
 * dempacking.cu:375-376), while N < n and time > (float)N*tnewpar/float(nplayer)
 * (:379-381), the next nplayer particles (the rest, at the end) join with
 * their injection states, no wall or pair history and zero displacement
 * since the list, and the step re-lists (:459-461): the re-list window
 * restarts there.  Forces, observables (packing fraction over the particles
 * in the system, mean CN = 2 contacts / N), dem_download_pairs and the window
 * kernels cover the N particles in the system; dem_download_state* returns
 * all n, those not yet poured in as injected.  A later upload ends the pour.
 * Layers join in the caller's order: on a context whose upload sorted the
 * particles by cell, dem_set_pour first puts them back (the state is kept,
 * the contact history restarts).
 * DEM_ERR_STATE before an upload or when a pour is already set (upload again
 * to start over); dem_adjoint_window refuses (DEM_ERR_STATE) until every
 * particle is in.  dem_active_count: N (n when not pouring). */
int dem_set_pour(dem_ctx* ctx, long long nplayer, double tnewpar, long long n_active);
int dem_active_count(dem_ctx* ctx, long long* n_active);

/* ---------------------------------------------------------------- adjoint --
 * Reverse mode of the step (force + walls + integrator) over a window; no
 * counterpart in the reference.  The forward runs nsteps from the current
 * state (saving a checkpoint every `checkpoint_every` steps), the objective
 * is evaluated at the final state, and the reverse sweep recomputes each
 * segment from its checkpoint.  Gradients are with respect to the contact
 * parameters (dem_contact layout; nu is not differentiated) and every radius.
 * nsteps must be a multiple of checkpoint_every, which must be a multiple of
 * relist_interval, and the call must start at a re-list boundary.  On return
 * the context holds the state at the end of the window. */
#define DEM_OBJ_PACKING    0   /* sum (4/3) pi r^3 / (Wx Wy max z)              */
#define DEM_OBJ_POTENTIAL  1   /* sum m z + sum (2/5) estar sqrt(R*) delta^2.5  */

typedef struct {
    double value;          /* objective at the end of the window              */
    dem_contact d_pp;      /* d objective / d particle-particle parameters    */
    dem_contact d_pw;      /* d objective / d particle-wall parameters        */
    double forward_ms;     /* device time of the checkpointed forward         */
    double adjoint_ms;     /* device time of the objective + recompute + reverse */
} dem_adjoint_result;

int dem_adjoint_window(dem_ctx* ctx, long long nsteps, int checkpoint_every, int objective,
                       dem_adjoint_result* out, double* d_radii /* host [n] or NULL */);
/* Frees the adjoint workspace (checkpoints, tape); dem_destroy does it too. */
int dem_adjoint_release(dem_ctx* ctx);

/* ============================================================================
 * 3. Host utilities (deck, initial states, reference output files)
 * ==========================================================================*/

/* hopp3d.inp deck as read at dempacking.cu:107-126, and the reduced-unit
 * constants derived at dempacking.cu:141-149,213-225. */
typedef struct {
    int iforcemode, ntot;
    double emod, vpois, denp, diam;
    double dt; unsigned int tstop;
    double dmt1, dmt2, thick, zht1, zht2;
    double vel0; int nrings;
    double ufricp, ufricw;
    double dampnp, damptp, dampnw, damptw, cdamp;
    double stiffness, dampcoeffn, dampcoefft;
    double upp, upw;
    /* derived (reduced units) */
    double emod_red, estarp, estarw;
    double world[3];          /* dmt2/diam, thick/diam, (zht1+zht2)/diam */
    double upp_red, upw_red;
} dem_deck;
int dem_read_deck(const char* path, dem_deck* out);
/* Material for the context API from a deck (pp and pw blocks). */
int dem_deck_material(const dem_deck* deck, dem_material* out);

/* Reduced-unit Hertz/restitution helpers.
 * dem_estar: (4/3)*emod_red/(2(1-nu^2)) with emod_red = 6E/(pi rho g d).
 * dem_damp_from_restitution: coefficient c with c*sqrt(6 m* E* sqrt(R* d))
 * equal to the viscous term of restitution e (E* = (3/4) estar). */
double dem_reduced_modulus(double E, double rho, double d);
double dem_estar(double E, double nu, double rho, double d);
double dem_damp_from_restitution(double e);

/* Initial states, reproducible from a 64-bit seed (SplitMix64).  Output is
 * host AoS pos[3n] and rad[n] in reduced units; world is the box.
 * Lattice: spacing a, nx*ny per layer centred in x,y, first layer z0, uniform
 * jitter +-jit, radius r (configuration of 2,000 spheres in a 20x20 box).
 * RSA: random sequential non-overlapping insertion with wall clearance r;
 * radii from dem_radius_* below.  Returns DEM_ERR_ARG when it cannot place. */
int dem_gen_lattice(long long n, double spacing, int nx, int ny, double z0, double jitter,
                    double radius, unsigned long long seed, double* pos, double* rad);
#define DEM_RADII_MONO       0  /* all r = a                                    */
#define DEM_RADII_LOGNORMAL  1  /* exp(ln a + b Z) truncated to [c, d]          */
#define DEM_RADII_BIDISPERSE 2  /* a and b, 1:1 by number, shuffled             */
int dem_gen_radii(long long n, int kind, double a, double b, double c, double d,
                  unsigned long long seed, double* rad);
int dem_gen_rsa(long long n, const double world[3], const double* rad,
                unsigned long long seed, double* pos);

/* Reference output files (formats of dempacking.cu:227-234,772-776,787-791,
 * 802,812-819,904-913). */
int dem_write_view(const char* path, const dem_deck* deck);
int dem_write_ppor(const char* path, long long it, long long n, long long pcntot,
                   double porosity, double packing, double avercn, double maxhz);
int dem_write_particles(const char* path, int zone, long long n, const double* pos,
                        const double* rad, double diam);
int dem_write_preflow(const char* path, long long it, long long n, long long itime,
                      const double* pos, const double* pdis, const double* angv);
int dem_write_timesteps(const char* path, double tret, long long it);
/* Reads preflow.dat as dem_write_preflow writes it (the reference's reader is
 * commented out, dempacking.cu:361-367).  pos == NULL: header only
 * (it, n, itime); else n particles into arrays of ncap particles (6 decimals
 * per value, as written). */
int dem_read_preflow(const char* path, long long* it, long long* n, long long* itime, double* pos,
                     double* pdis, double* angv, long long ncap);
int dem_write_finish(const char* jobfinished_path, const char* restart_path);

#ifdef __cplusplus
}
#endif
#endif /* DEM_B200_H */
