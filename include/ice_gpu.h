/*
 * ice_gpu.h -- C ABI of the B200 (sm_100a) solve stage of ICE's Eulerian
 * dispersed-phase time step.
 *
 * The Fortran driver keeps its INI registry, multi-block set-up, closure
 * selection and Tecplot/VTK I/O. After set-up it hands the library the
 * resolved parameters, the block metrics, the boundary table, the frozen gas
 * and the initial state; then each call of ice_gpu_step replaces
 *     call Explicit_Step(simulation%domain(lv))      (src/lib/driver/Wrap_Solve.f90:26)
 * for one or more time steps, with every array resident in HBM.
 *
 * Conventions
 *  - Every entry point returns 0 on success and a non-zero ICE_GPU_E* code on
 *    failure; ice_gpu_last_error() returns the message. Nothing traps: a
 *    failing state stops the step and is reported through the status word,
 *    as the reference's `error stop 1` sites would.
 *  - Indices in records are 1-based, as in the Fortran tables.
 *  - Host arrays use the Fortran layouts of the reference, so the driver can
 *    pass its own arrays with c_loc(); the library copies them and keeps no
 *    host pointer after a call returns.
 *  - One host thread per context; a context owns one CUDA stream.
 */
#ifndef ICE_GPU_H
#define ICE_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ICE_GPU_ABI_VERSION   1
#define ICE_GPU_MAX_FAMILIES  4
#define ICE_GPU_NCOND_MAX     12
#define ICE_GPU_NEP           8
#define ICE_GPU_REC_INTS      15   /* b i j k f type p bs is js ks fs partner owner cf */
#define ICE_GPU_REC_REALS     8    /* massflux velocity alpha beta temperature radius gfixed normal_dir */

/* Return codes */
#define ICE_GPU_OK             0
#define ICE_GPU_EINVAL         1   /* bad argument or inconsistent input */
#define ICE_GPU_ECUDA          2   /* CUDA runtime error */
#define ICE_GPU_ESTATE         3   /* the step stopped on a state the reference stops on */
#define ICE_GPU_ENOMEM         4
#define ICE_GPU_ENOTREADY      5   /* a required input has not been given */
#define ICE_GPU_EEXCH          6   /* the exchange hook of a split run reported a failure */

/* Status bits of ice_gpu_step_out.status (the reference's error stops) */
#define ICE_GPU_ST_NAN_STATE   1   /* NaN/Inf after an update   (Lib_Newstate.f90:189-193)  */
#define ICE_GPU_ST_BAD_RECON   2   /* unphysical first-order face (Mod_Fluxes.f90:238-241,
                                      Mod_BC_Fluxes.f90:95-98)                               */
#define ICE_GPU_ST_TIMEOUT     4   /* a bounded device wait gave up                          */

/* Closures (Assign_Setup.f90:104-117) */
#define ICE_CLOSURE_MK 1           /* rho u v w T n                                   (6) */
#define ICE_CLOSURE_IG 2           /* rho u v w P T n                                 (7) */
#define ICE_CLOSURE_AG 3           /* rho u v w P11 P12 P13 P22 P23 P33 T n          (12) */

/* Riemann solvers (Lib_Riemann.f90:30-57) */
#define ICE_RIEMANN_SAUREL  1
#define ICE_RIEMANN_RUSANOV 2
#define ICE_RIEMANN_HLLE    3

/* Limiters, in the order of assign_limiter (Lib_Limiters.f90:35-86); 0 is first order */
#define ICE_LIM_IORD       0
#define ICE_LIM_MINMOD     1
#define ICE_LIM_VANALBADA  2
#define ICE_LIM_VANLEER    3
#define ICE_LIM_OSPRE      4
#define ICE_LIM_UMIST      5
#define ICE_LIM_OSHER      6
#define ICE_LIM_SWEBY      7
#define ICE_LIM_MC         8
#define ICE_LIM_KOREN      9
#define ICE_LIM_SUPERBEE  10

/* Precision forms */
#define ICE_PREC_FP64      0       /* plain form: everything FP64                       */
#define ICE_PREC_FP32FLUX  1       /* reconstruction, Riemann fluxes and sources in FP32,
                                      RK accumulation, dt reduction and norms in FP64    */

/* One particle family: its closure, its Riemann solver, its frozen slots and
 * the constant-property material it is made of (condensed_phase_t,
 * src/lib/config/Config_Types_m.f90; ep packed as Setup_Materials.f90:152-160). */
typedef struct ice_gpu_family {
    int32_t closure;                    /* ICE_CLOSURE_*                                  */
    int32_t riemann;                    /* ICE_RIEMANN_*                                  */
    int32_t nfrozen;                    /* slots setup_freeze does not integrate          */
    int32_t frozen[ICE_GPU_NCOND_MAX];  /* their 1-based numbers                          */
    double  rho_al;                     /* material density [kg/m3]                       */
    double  cs_al;                      /* material specific heat [J/(kg K)]              */
    double  lv_al;                      /* latent heat [J/kg]                             */
    double  emiss;                      /* surface emissivity [-]                         */
    int32_t evap;                       /* 0 none, 1 d2, 2 CEM, 3 CEM-B, 4 ASM, 5 TC      */
    int32_t intf;                       /* 0 VLE, 1 Langmuir-Knudsen                      */
    int32_t liq;                        /* 0 ITC (P2T not supported: ICE_GPU_EINVAL)      */
    int32_t boil;                       /* 0 clamp (ZGR not supported: ICE_GPU_EINVAL)    */
    double  ep[ICE_GPU_NEP];            /* Mv Lv cpv Le Yinf LvMv/Ru 1/Tboil alphaE      */
} ice_gpu_family;

/* The resolved numerics of a run (obj_time_scheme, obj_space_scheme, obj_irs,
 * obj_sim_param, obj_io of the reference). */
typedef struct ice_gpu_params {
    int32_t nfam;                       /* ngroups                                        */
    int32_t ndir;                       /* 1, 2 or 3 (Mod_Metrics check_mesh_type)        */
    int32_t nrk;                        /* 1 euler, 2 RK2, 3 RK3                          */
    int32_t time_accurate;              /* 1: one global dt; 0: each cell its own dt      */
    double  cfl;
    double  dt_max;
    double  tau_factor;
    int32_t cfl_ramp_iter;
    int32_t limiter;                    /* ICE_LIM_*; 0 = first-order reconstruction      */
    int32_t shock_detector;             /* 1: Jameson sensor on density                   */
    int32_t irs;                        /* implicit residual smoothing (steady runs only) */
    double  irs_beta;
    int32_t coupled;                    /* one-way coupling to a frozen gas: sources on   */
    int32_t drag;                       /* 1..13, Lib_Drag.f90:19-79                      */
    int32_t heat;                       /* 1..8,  Lib_Heat.f90:18-64                      */
    int32_t blow;                       /* 0 none, 1 MHB98 f2                             */
    int32_t precision;                  /* ICE_PREC_*                                     */
    int32_t itermax;                    /* iterations of this call of the solver          */
    int32_t sol_diter;
    int32_t shell_diter;
    int32_t res_diter;
    int32_t no_realize;                 /* 1: the FP32-flux form skips its realizability
                                           correction of AG states (ice_gpu_step_out::
                                           nrealized); 0, the default, applies it         */
    double  time_threshold;
    double  res_threshold;
    double  sol_dtime;
    ice_gpu_family fam[ICE_GPU_MAX_FAMILIES];
} ice_gpu_params;

/* What one call of ice_gpu_step leaves for the driver (Explicit_Step's outputs). */
typedef struct ice_gpu_step_out {
    double  dtglobal;                   /* the last step's global dt                      */
    double  time;                       /* simulated time after the last step             */
    int32_t iter;                       /* grid%iter after the last step                  */
    int32_t todo;                       /* 1 continue, 2 output, 3 end (Mod_Explicit.f90:225-239) */
    int32_t status;                     /* ICE_GPU_ST_* bits                              */
    int32_t have_norm;                  /* residual[] holds the last step's norm          */
    int64_t nfloored;                   /* negative densities floored so far              */
    double  residual[5];                /* residual norm (rho, rho u, rho v, rho w, T)    */
    double  device_ms;                  /* device time of this call's steps (CUDA events on
                                           the context's stream)                          */
    int64_t nrealized;                  /* cell updates whose AG covariance the FP32-flux
                                           form's realizability correction made positive
                                           definite, so far (0 in the plain form)         */
} ice_gpu_step_out;

/* Training of the evaporation surrogate (ice_gpu_surrogate_train). */
typedef struct ice_gpu_surrogate_opts {
    int64_t  nsamples;                  /* training pairs drawn from the plain closure    */
    int32_t  epochs;
    int32_t  batch;
    double   lr;                        /* Adam's initial learning rate (cosine decay)    */
    double   jitter;                    /* spread of the sampled radius and speed (relative)
                                           and temperatures (x 20 K) around visited cells */
    uint64_t seed;
    double   val_frac;                  /* held-out fraction of the pairs                 */
} ice_gpu_surrogate_opts;

typedef struct ice_gpu_surrogate_report {
    double  train_loss;                 /* mean-square loss of the last 20 batches (standardised) */
    double  val_loss;                   /* the same on the held-out pairs                 */
    double  mdot_rel_median, mdot_rel_p99;   /* held-out relative error of the mass rate  */
    double  q_rel_median, q_rel_p99;         /* and of the heat rate                      */
    double  seconds;                    /* sampling and training                          */
    int64_t nsamples, steps;
    double  env_lo[7], env_hi[7];       /* the envelope of the seven inputs the network accepts */
} ice_gpu_surrogate_report;

typedef struct ice_gpu_ctx ice_gpu_ctx;

/* Set-up (after setup_freeze, Wrap_Setup.f90:121). dims: 3 ints per block.
 * replaces: allocate_data / Allocate_Block (driver/Mod_Allocate_Data.f90:8-133)
 * for the solve stage's arrays. */
int ice_gpu_create(const ice_gpu_params* params, int32_t nblocks, const int32_t* dims,
                   ice_gpu_ctx** ctx);

/* Metrics of block b (1-based), Fortran layouts of Allocate_Block:
 *   face_d : per face 4 doubles (N(3), A), dir(1)%f(0:ni,1:nj,1:nk),
 *            dir(2)%f(1:ni,0:nj,1:nk), dir(3)%f(1:ni,1:nj,0:nk)
 *   vol    : (1:ni,1:nj,1:nk)
 *   dl     : 3 doubles per cell on (0:ni+1,0:nj+1,0:nk+1)
 *   M      : 9 doubles per cell (column-major c(3,3)) on (0:ni+1,0:nj+1,0:nk+1)
 * replaces: setup_metrics' results (numerics/space/Mod_Metrics.f90:19-60). */
int ice_gpu_set_block(ice_gpu_ctx* ctx, int32_t b, const double* face1, const double* face2,
                      const double* face3, const double* vol, const double* dl, const double* M);

/* The whole boundary table in table order (grid%bc), ICE_GPU_REC_INTS ints and
 * ICE_GPU_REC_REALS reals per record, partner/owner/cf as Pair_Connections left
 * them. The library builds the per-family record lists, the boundary cells with
 * their records in face order and the connection owners from it.
 * replaces: build_local_bc_index (parallel/Mod_GhostExchange.f90:103-172). */
int ice_gpu_set_records(ice_gpu_ctx* ctx, int32_t nrec, const int32_t* rec, const double* inlet);

/* The donors of the table's chimera records (code 102), after ice_gpu_set_records: for each
 * record of the table in table order, nchi[2n] and nchi[2n+1] donors of ghost layers 1 and 2
 * (0 and 0 unless the record is 102; at least one each if it is), then every donor in the
 * same order, donor[4s..4s+3] = block, i, j, k (1-based, an interior cell) and weight[s].
 * Each ghost cell is the weighted sum of its donors' conservative states (ghost_chimera,
 * numerics/space/Lib_Ghost.f90:439-466); a step refuses to run while 102 records lack donors.
 * replaces: the chimera payload of read_bc (io/IO_BC.f90:209-236) stored in ICE_bc_type%ni,
 * donorID, volume_fraction (base/Advanced_Types_m.f90:29-31). */
int ice_gpu_set_chimera(ice_gpu_ctx* ctx, int32_t nrec, const int32_t* nchi, const int32_t* donor,
                        const double* weight);

/* Frozen gas of block b: prim5 (5,ni,nj,nk) = rho u v w T, then R, gamma, k, mu (ni,nj,nk).
 * replaces: setup_gas (driver/Mod_Phase.f90:11-63). */
int ice_gpu_set_gas(ice_gpu_ctx* ctx, int32_t b, const double* prim5, const double* R,
                    const double* gam, const double* k, const double* mu);

/* The coupler's imports into family p (1-based) of block b: imports (ncond, ni, nj, nk), the rates
 * that the coupler's add_birth_rate, add_absorption_rate and add_removal_rate accumulate in
 * ICE_cond_phase_type%imports (coupling/Mod_Exchange.f90:270-390); NULL sets the block's rates to
 * zero. From the first call on, every step of the family adds imports * dt to the residual
 * (add_births) and bounds its steps as bound_empty_dt and bound_removal_dt do.
 * replaces: add_births (numerics/time/explicit/Lib_Residual.f90:164-210), bound_empty_dt and
 * bound_removal_dt (numerics/time/Mod_dt.f90:134-242) for a coupled family. */
int ice_gpu_set_imports(ice_gpu_ctx* ctx, int32_t b, int32_t p, const double* imports);

/* Two-way coupling on (on != 0) or off: every stage then adds its source to the step's running sum,
 * weighted as the update weighs the stages, for ice_gpu_exchange_rate.
 * replaces: add_stage_source and hand_step_source (numerics/time/explicit/Mod_Explicit.f90:257-300)
 * of a twcoupled run. */
int ice_gpu_set_exchange(ice_gpu_ctx* ctx, int32_t on);

/* What family p (1-based) gave the gas from every cell of block b over the last step, per unit volume
 * and time: x (5, ni, nj, nk) = mass, momentum (3), energy (no burning family: nothing is generated
 * and there is no heat of reaction).
 * replaces: exchange_rate (coupling/Mod_Exchange.f90:60-78). */
int ice_gpu_exchange_rate(ice_gpu_ctx* ctx, int32_t b, int32_t p, double* x);

/* State of family p (1-based) in block b: prim (ncond, 1-gc:ni+gc, 1-gc:nj+gc, 1-gc:nk+gc),
 * gc = 2; inj the injected-ghost flags on the same cells (NULL: all false).
 * replaces: setup_cond's result (driver/Mod_Phase.f90:66-124). */
int ice_gpu_upload_state(ice_gpu_ctx* ctx, int32_t b, int32_t p, const double* prim,
                         const uint8_t* inj);

/* The state back in the same layout (interior cells exact; ghost cells hold the
 * last fill). Called before Write_Solution (Wrap_Postprocess.f90:120-196). */
int ice_gpu_download_state(ice_gpu_ctx* ctx, int32_t b, int32_t p, double* prim);

/* Simulated time and iteration count (a restart, or a second call of the solver). */
int ice_gpu_set_time(ice_gpu_ctx* ctx, double time, int32_t iter, int32_t iter_from_call);

/* The unit of res-threshold: the first non-zero density residual of a steady run (0 until one has
 * come; set from a restart's counters, read to write them).
 * replaces: obj_sim_param%res_reference (config/Config_Types_m.f90:45; driver/Wrap_Setup.f90:197-215,
 * io/IO_Solution.f90:244,440). */
int ice_gpu_set_res_reference(ice_gpu_ctx* ctx, double ref);
int ice_gpu_get_res_reference(ice_gpu_ctx* ctx, double* ref);

/* nsteps time steps. replaces: call Explicit_Step(grid) (driver/Wrap_Solve.f90:26),
 * numerics/time/explicit/Mod_Explicit.f90:11-245. Returns ICE_GPU_ESTATE when a
 * step ended on a state the reference stops on (out->status says which). A steady run with
 * res_threshold > 0 takes the residual norm after every step (out->residual) and the call ends at
 * the step whose density residual is at most res_threshold times the run's first non-zero one
 * (out->todo = 3), as the driver's loop ends on TODO = 3. Returns ICE_GPU_ENOTREADY, before any
 * launch, when the set-up is incomplete: a block without metrics, no boundary table, chimera records
 * without donors, or gas missing where it is read (a coupled run, or a 401 or 403 inlet, with a block
 * that ice_gpu_set_gas has not filled). */
int ice_gpu_step(ice_gpu_ctx* ctx, int32_t nsteps, ice_gpu_step_out* out);

/* nsteps time steps for a driver that keeps the state on the host. prim_in[(b-1)*nfam + (p-1)]
 * holds family p of block b in the layout of ice_gpu_upload_state, and prim_out the same for the
 * state after the steps (prim_out may equal prim_in). The result is that of upload_state for every
 * block and family, then ice_gpu_step(nsteps), then download_state for every block and family. Here
 * the uploads, the steps and each family's download overlap, so the call takes less time than those
 * calls one after another. Page-locked host arrays let the copies run at full speed.
 * replaces: call Explicit_Step(grid) (driver/Wrap_Solve.f90:26) with the state kept in the
 * driver's arrays. */
int ice_gpu_step_host(ice_gpu_ctx* ctx, int32_t nsteps, const double* const* prim_in,
                      double* const* prim_out, ice_gpu_step_out* out);

/* The residual norm of the last step: total[5], and fam[5*nfam] per family (may be NULL).
 * replaces: residual_norm (diagnostic/Mod_Diagnostic.f90:22-83). */
int ice_gpu_residual_norm(ice_gpu_ctx* ctx, double* total, double* fam);

/* The residual-norm sums of one block of one family for a caller that cannot allocate device
 * memory: a driver whose device memory all belongs to the host application's own allocator (a
 * coupler inside a gas solver with a fixed device-memory budget, a Fortran/OpenACC runtime that
 * owns the state arrays) and so may create no solve context, whose set-up allocates. No counterpart
 * in the reference: it is the per-block part of residual_norm without a context.
 * prim_new, prim_old: DEVICE arrays of the block in the driver's layout prim(nc, 1-gc:ni+gc,
 * 1-gc:nj+gc, 1-gc:nk+gc), gc = 2; t_slot the 1-based temperature slot (nbase - 1); dims ni nj nk.
 * sums[5] (host): the sums over interior cells of (new - old)^2 of rho, u, v, w, T; the residual
 * norm is the square root of their sum over blocks and families (the same bits as
 * ice_gpu_residual_norm for the same states). stream: a cudaStream_t, or NULL.
 * It allocates nothing: its scratch is a static device array of 4096 x 5 partial sums (plus 5),
 * which every GPU that loads the library holds until exit; a block of more than 8,388,608 cells is
 * refused with ICE_GPU_EINVAL. The first call in a CUDA context (the device's primary context, or
 * one the caller's runtime made) looks the array up in that context (make it before any stream
 * capture). Each call ends by copying the five sums to the host and synchronising its stream. Every
 * call overwrites all the scratch it reads, so nothing carries over between calls; two calls that
 * overlap on the GPU (other streams) share the array and race.
 * Errors: a message in err[errlen]. */
int ice_gpu_residual_sq_noalloc(const double* prim_new, const double* prim_old, int32_t nc,
                                int32_t t_slot, const int32_t* dims, double* sums, void* stream,
                                char* err, int32_t errlen);

/* The evaporation surrogate of family p (FP32-flux form, coupled runs): draws o->nsamples inputs
 * around the cells of the current state, evaluates the plain FP64 closure on them (evaporation with
 * its interface model, the heat correlation, override or blowing: compute_source_,
 * Mod_Sources.f90:520-551), trains a 7 -> 128 x 4 -> 2 SiLU network on them with the library's own
 * FP32 forward, backward and Adam kernels, and switches the family's source to it: BF16 tensor-core
 * inference, with the plain closure for every cell outside the training envelope or whose rates fail
 * the closure's own equations by more than 1e-3. No counterpart in the reference (its closure is
 * always evaluated); it replaces the iterative part of the evaporation source. */
int ice_gpu_surrogate_train(ice_gpu_ctx* ctx, int32_t p, const ice_gpu_surrogate_opts* opts,
                            ice_gpu_surrogate_report* report);

/* Switches family p between the trained surrogate (on) and the plain closure (off). */
int ice_gpu_surrogate_enable(ice_gpu_ctx* ctx, int32_t p, int32_t on);

/* Cumulative counts of the surrogate source: counts[0] cells evaluated, counts[1] of them outside
 * the envelope, counts[2] of them failing the closure check (both ran the plain closure). */
int ice_gpu_surrogate_stats(const ice_gpu_ctx* ctx, int64_t* counts);

/* Checks of the surrogate's kernels on host arrays (no context): the loss (mean-square over n x 2
 * standardised targets t) and its gradient with respect to the FP32 parameters w of the training
 * kernels, for n standardised inputs x (n x 7); and the BF16 tensor-core forward pass y (n x 2).
 * No counterpart in the reference. */
int ice_gpu_mlp_grad(const float* w, const float* x, const float* t, int32_t n, float* grad, float* loss);
int ice_gpu_mlp_infer(const float* w, const float* x, int32_t n, float* y);

/* A runtime re-read of input.ini (Wrap_Postprocess.f90:255 -> Read_Ini.f90:61): the
 * numerics may change between steps; nfam, closures and ndir may not. */
int ice_gpu_update_params(ice_gpu_ctx* ctx, const ice_gpu_params* params);

/* The message of the last failing call on ctx (or of ice_gpu_create when ctx is NULL). */
int ice_gpu_last_error(const ice_gpu_ctx* ctx, char* buf, int32_t buflen);

int ice_gpu_destroy(ice_gpu_ctx* ctx);

/* Host-only: partner, owner and face number of every connection record (101/201)
 * of a boundary table in table order, written into fields 13..15 of rec.
 * replaces: Pair_Connections (io/IO_BC.f90:360-510). ngroups families, the
 * records of boundary cell n and family p at position (n-1)*ngroups + p. */
int ice_gpu_pair_connections(int32_t nblocks, const int32_t* dims, int32_t ngroups,
                             int32_t nrec, int32_t* rec, char* err, int32_t errlen);

/* Debug / parity: the index maps the library built from the boundary table.
 * For family p: nbcell boundary cells, first[nbcell+1] (1-based into recs),
 * recs[] (1-based record numbers in face order), nown owners own[] (1-based).
 * Pass NULL arrays to query the counts. replaces nothing: it exposes
 * grid%bcells(p) and grid%conn(p)%own for comparison with the reference's. */
int ice_gpu_index_maps(const ice_gpu_ctx* ctx, int32_t p, int32_t* nbcell, int32_t* first,
                       int32_t* nrecs, int32_t* recs, int32_t* nown, int32_t* own);

/* ---- The block split over ranks (one GPU per rank) --------------------------------------------
 * replaces: the MPI block decomposition of parallel/Mod_MPI.f90:109-183 (blocks per rank) and the
 * exchanges of parallel/Mod_GhostExchange.f90:737-893 (remote source cells of the ghost layers,
 * connection fluxes owner -> partner, partner Jameson weights), with the min-reduction of the step's
 * dt (Mod_Explicit.f90:67-73) and the sum of the residual norm's partial sums.
 *
 * Every rank creates a context of the whole case (every block's geometry, records and gas), then
 * ice_gpu_set_partition names the blocks it steps; it keeps the other blocks' state only where its
 * ghost layers read them. ice_gpu_set_halo gives, per family and kind, the entries this rank sends
 * and receives, in buffer order, per peer one after the other. At each exchange point the step packs
 * the send buffer, calls the hook, and unpacks the receive buffer the hook filled. Every rank calls
 * the hook at the same points, in the same order: a hook over MPI or torch.distributed matches them.
 * ice_gpu_residual_norm is then collective too. Imports, chimera records and IRS are refused. */
#define ICE_GPU_HALO_CELLS 0   /* entries (b, i, j, k), 1-based; nc doubles each: the cell's state      */
#define ICE_GPU_HALO_BETA  1   /* entries (b, i, j, k); one double each: the cell's Jameson weight     */
#define ICE_GPU_HALO_FLUX  2   /* entries (cf, 0, 0, 0): nc doubles each, a connection face's flux       */
#define ICE_GPU_HALO_DT    3   /* the hook's reduction: the minimum over ranks of 1 double             */
#define ICE_GPU_HALO_NORM  4   /* the hook's reduction: the sum over ranks of 5 nblocks nfam doubles   */

/* The exchange: kind, 1-based family (0 for DT and NORM), the packed send buffer of nsend doubles
 * and the receive buffer of nrecv doubles to fill (host memory). For DT and NORM the hook writes the
 * reduction of every rank's send buffer into recv. Returns 0, or non-zero to stop the step with
 * ICE_GPU_EEXCH. */
typedef int32_t (*ice_gpu_exchange_fn)(void* user, int32_t kind, int32_t family, int64_t nsend,
                                       const double* send, int64_t nrecv, double* recv);

/* owned[nblocks]: 1 for a block this rank steps, 0 otherwise (default: every block). */
int ice_gpu_set_partition(ice_gpu_ctx* ctx, const int32_t* owned);

/* The lists of one kind (HALO_CELLS, BETA or FLUX) of family p: send[4 nsend], recv[4 nrecv]. */
int ice_gpu_set_halo(ice_gpu_ctx* ctx, int32_t kind, int32_t p, int32_t nsend, const int32_t* send,
                     int32_t nrecv, const int32_t* recv);

/* The hook a split step calls at its exchange points (user is passed back). */
int ice_gpu_set_exchange_hook(ice_gpu_ctx* ctx, ice_gpu_exchange_fn fn, void* user);

/* Measurement: device time [ms] of the kernels of the last ice_gpu_step, by kernel
 * class (0 dt, 1 ghost, 2 beta, 3 bound, 4 stage, 5 irs, 6 norm), and the
 * number of kernels launched. Filled only when the context was made with
 * profiling on (ice_gpu_set_profiling). */
int ice_gpu_set_profiling(ice_gpu_ctx* ctx, int32_t on);
int ice_gpu_kernel_times(const ice_gpu_ctx* ctx, double* ms, int32_t nclass, int64_t* nlaunch);

#ifdef __cplusplus
}
#endif

#endif /* ICE_GPU_H */
