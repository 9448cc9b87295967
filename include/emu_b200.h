/*
 * emu_b200.h -- C ABI of the B200 implementation of Emu's per-step particle
 * evolution path (deposit_to_mesh -> interpolate_rhs_from_mesh -> Runge-Kutta
 * stage update -> periodic wrap -> Renormalize -> compute_dt).
 *
 * Plain C types only: pointers, sizes, status codes.  Every entry point
 * returns EMU_OK (0) or an OR of EMU_ERR_* bits and never aborts the process;
 * emu_last_error() gives the message.  Reference functions are cited as
 * file:line in the Emu source tree (AMReX-Astro/Emu).
 *
 * Particle records (host side) are FP64 rows of emu_nreal(nflavors) values:
 *   pos_x, pos_y, pos_z, then the PIdx attributes
 *   time,x,y,z,pupx,pupy,pupz,pupt,N,L,f..,Nbar,Lbar,f..bar
 * (Source/FlavoredNeutrinoContainer.H:12-26 + generated H_fill), i.e. the
 * real-component order of the reference's particle output
 * (Scripts/visualization/amrex_plot_tools.py:12-90).
 *
 * Mesh output is emu_ncomp(nflavors) planes of ncell[0]*ncell[1]*ncell[2]
 * FP64 values, i fastest, in GIdx order (Source/Evolve.H:11-27):
 *   rho,T,Ye, N,Nbar,Fx,Fxbar,Fy,Fybar,Fz,Fzbar (each nflavors^2 reals).
 */
#ifndef EMU_B200_H_
#define EMU_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EMU_B200_ABI_VERSION 1

/* status bits */
#define EMU_OK           0
#define EMU_ERR_TRACE    1     /* Renormalize: |trace-1| > 100*maxError   (generate_code.py:404-409) */
#define EMU_ERR_NEGDIAG  2     /* Renormalize: diagonal < -100*maxError  (generate_code.py:418-423) */
#define EMU_ERR_LENGTH   4     /* Renormalize: |length-L| > 100*maxError  (generate_code.py:433-438) */
#define EMU_ERR_DT       8     /* compute_dt: no limiter active           (Evolve.cpp:76-86)  */
#define EMU_ERR_ARG      16    /* invalid argument */
#define EMU_ERR_CUDA     32    /* CUDA runtime failure (no device, launch error, ...) */
#define EMU_ERR_STATE    64    /* call out of order (e.g. no particles loaded) */
#define EMU_ERR_IO       128   /* file I/O */
#define EMU_ERR_PARSE    256   /* inputs file */
#define EMU_ERR_NOMEM    512   /* allocation failed */
#define EMU_ERR_LIMIT    1024  /* size beyond a documented limit */
#define EMU_ERR_TIMEOUT  2048  /* a bounded device-side wait gave up (results of that step are invalid) */

/* arithmetic of the path */
#define EMU_PREC_FP64    0     /* FP64 throughout (the reference's PRECISION=DOUBLE) */
#define EMU_PREC_MIXED   1     /* FP32 interpolation/potentials/commutator (the
                                  RHS), int64 fixed-point deposit, FP64 rho
                                  accumulation and renormalisation */

/*
 * Run parameters.  Mirrors TestParams (Source/Parameters.H:11-132) in the
 * reference's internal units: CGS, masses in grams, angles in radians (the
 * inputs file's eV and degrees are converted by emu_parse_inputs exactly as
 * Parameters.H:81-97 does).  The first five fields are the reference's
 * compile-time choices (NUM_FLAVORS, SHAPE_FACTOR_ORDER, PRECISION) and the
 * integrator keys (integration.type, integration.rk.type).
 */
typedef struct emu_params {
    int nflavors;            /* 2 or 3 */
    int shape_order;         /* 0, 1 or 2 */
    int precision;           /* EMU_PREC_FP64 or EMU_PREC_MIXED */
    int integration_type;    /* 0 forward Euler, 1 explicit Runge-Kutta */
    int rk_type;             /* 2 trapezoid, 3 SSPRK3, 4 classical RK4 */

    int ncell[3];
    int nppc[3];
    int nphi_equator;
    double Lx, Ly, Lz;
    int max_grid_size;
    int nsteps;
    double end_time;
    int write_plot_every;
    int write_plot_particles_every;
    double rho_in, Ye_in, T_in;
    int simulation_type;
    double cfl_factor, flavor_cfl_factor, max_adaptive_speedup;
    int do_restart;
    char restart_dir[512];
    double maxError;
    double mass1, mass2, mass3;
    double theta12, theta13, theta23;
    double alpha1, alpha2, deltaCP;
    int st3_wavelength_fraction_of_domain;
    double st3_amplitude;
    double st4_ndens, st4_theta, st4_phi, st4_fluxfac;
    double st4_ndensbar, st4_thetabar, st4_phibar, st4_fluxfacbar;
    double st4_amplitude;
    double st5_nnue, st5_nnua, st5_nnux;
    double st5_fxnue, st5_fxnua, st5_fxnux;
    double st5_fynue, st5_fynua, st5_fynux;
    double st5_fznue, st5_fznua, st5_fznux;
    double st5_amplitude;

    /* extensions of this implementation */
    int direction_generator; /* 0: uniform_sphere_xyz ring generator (Init.cpp:9-37),
                                1: Fibonacci sphere with ndirections points */
    int ndirections;
    uint64_t seed;           /* counter-based RNG seed for sim types 4 and 5
                                (the reference seeds from the clock, main.cpp:240) */
    int resort_interval;     /* steps between on-device cell re-sorts (0 = never,
                                < 0 = automatic: every step for 3D stencils,
                                every 16 steps otherwise; default -1) */
    int fused;               /* RK4 kernels: 1 (default) one fused kernel per stage, a CUDA
                                graph per step; 2: one cooperative launch per step when the
                                grid fits on the GPU at once (FP64), else as 1; 0: unfused */
} emu_params;

/* summary of a device-resident run (emu_evolve) */
typedef struct emu_run_info {
    int steps_done;          /* steps completed by this call */
    int status;              /* OR of EMU_ERR_* raised on the device */
    int64_t bad_particle;    /* load index of the first particle that failed Renormalize, or -1 */
    double time;             /* integrator time after the last completed step */
    double dt_next;          /* timestep the next step would take (compute_dt on the last stage mesh) */
} emu_run_info;

typedef struct emu_context emu_context;

/* ---- sizes ---- */
int emu_nattribs(int nflavors);        /* PIdx::nattribs: 20 or 30 */
int emu_nreal(int nflavors);           /* 3 + nattribs */
int emu_ncomp(int nflavors);           /* GIdx::ncomp: 35 or 75 */
int emu_abi_version(void);

/* ---- configuration (host only, no GPU needed) ---- */
/* Defaults for every field (the values of Emu's sample inputs where one exists). */
void emu_params_default(emu_params* p);
/* Reads an inputs file plus "key=value" overrides with ParmParse syntax and
 * unit conversion (replaces TestParams::Initialize, Parameters.H:52-131).
 * Every key the reference requires is required here too. */
int emu_parse_inputs(const char* path, int n_overrides, const char* const* overrides,
                     emu_params* out, char* errbuf, size_t errlen);
/* Initial particles on the host (replaces FlavoredNeutrinoContainer::InitParticles,
 * FlavoredNeutrinoContainerInit.cpp:136-661).  With out == NULL only *n_out is set. */
int emu_init_particles(const emu_params* p, double* out, int64_t capacity, int64_t* n_out);
/* InitParticles on the device: the particles emu_init_particles would
 * return, generated in device memory and loaded into ctx (replaces
 * emu_init_particles + emu_load_particles without the host round trip).
 * Bit-identical records except where simulation types 3 and 5 evaluate
 * sin / exp.  A context attached to a communicator generates the particles
 * of global indices rank, rank + nranks, ... (its shard). */
int emu_init_particles_device(emu_context* ctx);
/* Vvac_max of a particle set (FlavoredNeutrinoContainerInit.cpp:657-660). */
int emu_vvac_max(const emu_params* p, const double* records, int64_t n, double* out);

/* ---- context (needs a CUDA device) ---- */
/* Creates the device context; the caller owns it.  Different contexts may be
 * driven from different host threads at once (one thread per context); the
 * library serialises its allocations and graph captures internally and makes
 * no device-wide synchronisation.  One context is not thread safe. */
int emu_create(const emu_params* p, emu_context** out);
void emu_destroy(emu_context* ctx);
/* Launch all work of this context on a caller-provided cudaStream_t (NULL =
 * the context's own stream). */
int emu_set_stream(emu_context* ctx, void* cuda_stream);
int emu_synchronize(emu_context* ctx);

/* Upload particle records (host memory).  Replaces InitParticles/Restart as the
 * source of the container; particles are cell-sorted on the device.  Returns
 * once the records have been copied (the buffer may be reused); the sort and
 * the deposit run on in the context's stream. */
int emu_load_particles(emu_context* ctx, const double* records, int64_t n);
/* Download particle records in load order. */
int emu_get_particles(emu_context* ctx, double* records, int64_t n);
int emu_num_particles(const emu_context* ctx, int64_t* n);

/* deposit_to_mesh (Evolve.H:31 / Evolve.cpp:91-126) of the current particles */
int emu_deposit(emu_context* ctx);
/* The current mesh (rho,T,Ye and the last deposit), GIdx planes.  After
 * steps: the deposit of the last step's stage-4 state, as the reference's
 * state MultiFab holds it.  (Mixed precision: EMU_ERR_STATE after a step
 * timed by emu_profile_step, which keeps only the layout stage 4 reads.) */
int emu_get_mesh(emu_context* ctx, double* out);
/* interpolate_rhs_from_mesh (Evolve.H:33 / Evolve.cpp:128-176): the time
 * derivative of every attribute of every particle, from the current mesh,
 * written as particle records in load order (positions copied through). */
int emu_interpolate_rhs(emu_context* ctx, double* rhs_records);
/* FlavoredNeutrinoContainer::Renormalize (FlavoredNeutrinoContainer.H:92). */
int emu_renormalize(emu_context* ctx, int64_t* bad_particle);
/* compute_dt (Evolve.H:29 / Evolve.cpp:22-89) on the current mesh. */
int emu_compute_dt(emu_context* ctx, double* dt);
/* One integrator step of length dt (TimeIntegrator::advance with
 * ApplyFlavoredNeutrinoRHS, FlavoredNeutrinoContainer.H:33-47) followed by the
 * post-timestep hook (SyncLocation, periodic Redistribute, Renormalize,
 * main.cpp:155-173).  Afterwards the current mesh is the last stage deposit. */
int emu_step(emu_context* ctx, double dt, int64_t* bad_particle);
/* The evolve_flavor loop (main.cpp:118,206,213): deposit, compute_dt, then up
 * to nsteps steps (stopping at end_time, dt clipped to land on it), with dt
 * recomputed on the device from each step's last stage mesh.  Runs without
 * host synchronisation between steps.  start_time is the integrator time of
 * the loaded particles. */
int emu_evolve(emu_context* ctx, int nsteps, double start_time, double end_time, emu_run_info* info);
/* emu_evolve in three parts, for callers that pipeline work on the stream:
 * begin = deposit + initial compute_dt on the device; steps = enqueue that
 * many steps (each a CUDA graph launch, no host synchronisation); end =
 * synchronise and report.  Steps past max_steps or end_time do no work. */
int emu_evolve_begin(emu_context* ctx, double start_time, double end_time, int max_steps);
/* Mixed precision without the adaptive timestep branch (max_adaptive_speedup
 * <= 1): the steps of one call but the last (and the last of the run) keep
 * their stage-4 mesh only in the layout stage 4 interpolates, plus the
 * diagonal N_ii that compute_dt reads, none of which a caller can read
 * before the call returns; the results do not depend on how a run is split
 * into calls. */
int emu_evolve_steps(emu_context* ctx, int nsteps);
int emu_evolve_end(emu_context* ctx, emu_run_info* info);
/* Limit of the bounded grid-barrier waits of this context's cooperative
 * kernels (the whole-step kernel of fused = 2 and the adjoint's segment
 * kernels), in polls of a 64 ns sleep; polls < 0 restores the default
 * (2^22).  A wait that runs out sets EMU_ERR_TIMEOUT in the run's status and
 * lets the kernel finish (the step's results are then invalid); the next
 * emu_evolve_begin or emu_load_particles resets the barrier.  No
 * counterpart in the reference (its steps have no device-side waits);
 * tests use a limit of 0 to make a wait run out. */
int emu_set_wait_limit(emu_context* ctx, int64_t polls);
/* Overwrite a device buffer (bytes, multiple of 8) on the context's stream;
 * benchmarks use it to evict the L2 cache between timed steps. */
int emu_flush_l2(emu_context* ctx, void* device_buffer, int64_t bytes);
/* One device-resident step (as a step inside emu_evolve_steps(ctx, n > 1))
 * launched kernel by kernel with a CUDA event pair around each launch on the
 * context stream.
 * kernel_ms[i] receives the duration of kernel i in launch order (the RK
 * stages, with the mixed path's finalize kernel before each; stage 4 also
 * reduces compute_dt), then, when a re-sort follows the step, the whole
 * re-sort (keys, radix sort, gather, and the deposit of the new state that
 * stage 4 then leaves out, as emu_evolve_steps does) as one more entry;
 * *nkernels their count (at most 9).  Call after emu_evolve_begin. */
int emu_profile_step(emu_context* ctx, float* kernel_ms, int max_kernels, int* nkernels);

/* Plotfile (IO.cpp:11-38): mesh plotfile pltNNNNN plus, when
 * write_particles != 0, the particle checkpoint pltNNNNN/neutrinos. */
int emu_write_plotfile(emu_context* ctx, const char* dir, double time, int step, int write_particles);
/* The same plotfile from host arrays (mesh as emu_get_mesh returns it,
 * records may be NULL): host only, no GPU needed. */
int emu_write_plotfile_host(const emu_params* p, const char* dir, double time, int step, const double* mesh,
                            const double* records, int64_t n);
/* Particle checkpoint reader (RecoverParticles, IO.cpp:40-63): host only. */
int emu_read_particles(const char* plotfile_dir, int nflavors, double* out, int64_t capacity,
                       int64_t* n_out, double* time, int* step);

/* Message of the last failure on this context (or of the last host-only call
 * when ctx is NULL). */
int emu_last_error(const emu_context* ctx, char* buf, size_t len);

/*
 * deposit_to_mesh for callers that cannot allocate device memory.  No
 * counterpart in the reference: its deposit writes into an AMReX MultiFab
 * the caller already owns.  Some host programs cannot let a library call
 * cudaMalloc: one that hands all device memory to its own pool allocator at
 * start-up has nothing left to allocate from, and a time-critical step loop
 * cannot afford cudaMalloc/cudaFree (cudaFree synchronises the whole
 * device).  This entry point allocates nothing.  Inputs and outputs are
 * device memory owned by the caller:
 *   d_records   n particle records (rows of emu_nreal(nflavors) FP64, the
 *               emu_load_particles layout, in any order), on the device
 *   d_mesh_out  emu_ncomp(nflavors) x ncells FP64 in emu_get_mesh layout
 * Its only scratch, the cell-major accumulation mesh, is a fixed array of
 * 2^19 doubles (4 MiB) compiled into the library; ncells * 8 * nflavors^2
 * must not exceed it (EMU_ERR_LIMIT otherwise).  Every GPU that loads the
 * library keeps the array until the process exits.  The first call in a
 * device context (and again after a device reset) looks up the array's
 * device address with cudaGetSymbolAddress, with that device current; make
 * that first call before any stream capture.  All calls share the array and
 * each call clears it first, so calls that overlap on the GPU (different
 * streams, threads or processes on one device) race and must be serialised
 * by the caller.  Work is enqueued on `stream` (a cudaStream_t, NULL = the
 * legacy default stream); the call does not synchronise.
 * Errors: emu_last_error(NULL, ...).
 */
int emu_deposit_noalloc(const emu_params* p, const double* d_records, int64_t n, double* d_mesh_out,
                        void* stream);

/*
 * Discrete adjoint of the FP64 RK4 evolution.  No counterpart in the
 * reference (it has no derivatives).  Arrays are host memory in load order:
 * lam_f rows hold dJ/d(the 2 nflavors^2 flavor reals of a record, nu then
 * nubar, in the record's f order); lam_N rows hold (dJ/dN, dJ/dNbar).
 *
 * emu_adjoint_forward: nsteps device-resident RK4 steps from the loaded
 * state with the configured timestep rule, recording every step's dt (into
 * dts when not NULL) and a checkpoint of (f, x) every checkpoint_interval
 * steps.  Particles keep their order (no re-sort) during a recorded run.
 * Requires precision FP64, integration_type 1, rk_type 4, fused >= 1.
 *
 * emu_adjoint_objective: J = sum over cells |N_emu|^2 / V_cell of the
 * current state (N_emu: the neutrino e-mu off-diagonal number deposited in
 * a cell; J is the domain integral of |n_emu|^2) and, when the pointers are
 * not NULL, dJ/df (n x 2nf^2) and dJ/d(N, Nbar) (n x 2) of that state.
 *
 * emu_adjoint_backward: given dJ/df of the final state of the recorded run
 * (lam_f_final, n x 2nf^2) and optionally dJ/d(N, Nbar) taken at the final
 * state (lam_N_final, n x 2, NULL = 0), the gradient with respect to the
 * run's initial f (lam_f0) and N, Nbar (lam_N0), with the recorded dt held
 * fixed.  When the states, stage states and meshes of every step of the run
 * fit the budget below (and, two flavors, the grid is co-resident), the
 * recorded forward stores them and the backward recomputes nothing
 * (environment variable EMU_ADJOINT_FULL_STORE=0 turns this off).  Otherwise
 * it recomputes each checkpoint segment from its checkpoint; the stage
 * states and meshes of a whole segment are kept when they fit a budget
 * (a quarter of the free device memory, at most 16 GiB; environment variable
 * EMU_ADJOINT_STORE_MAX_BYTES overrides it), else each step's stages are
 * recomputed before its backward step.  In that per-step mode the states of
 * every step of a segment are kept, or, when the checkpoints and those
 * states would not fit in the free device memory, sub-checkpoints inside
 * a segment held in J + interval / J segment slots, J =
 * ceil(sqrt(checkpoint_interval)) (each step is recomputed once more;
 * environment variable EMU_ADJOINT_SUBCHECKPOINT sets J, and
 * EMU_ADJOINT_SEG_SLOTS lowers the slot count, for tests).  With re-sorts,
 * the per-step mode also keeps each step's stage meshes when the free
 * memory allows (EMU_ADJOINT_STORE_MESHES=0 turns that off).  The context's
 * particle state is unchanged.
 *
 * emu_adjoint_reserve: allocates the checkpoint and work storage of a
 * recorded run of nsteps with this checkpoint_interval up front (what
 * emu_adjoint_forward would allocate), so that a timed or repeated run does
 * no allocation.  Optional outputs: the device bytes held, how stage states
 * are kept (2: every step of the run, stored by the recorded forward; 1:
 * recomputed and kept per segment; 0: recomputed per step), and the
 * sub-checkpoint spacing (0 = none).
 */
/*
 * Particle sharding over GPUs (one process per GPU).  No counterpart in the
 * reference, which distributes boxes of cells over MPI ranks.  Each rank
 * creates its context, attaches it to a communicator, then loads its own
 * disjoint subset of the particles; the mesh is replicated and every deposit
 * is summed over the ranks (NCCL all-reduce on the context's stream) before
 * any stage reads it, so every rank computes the same compute_dt and takes
 * the same steps.  Vvac_max and the mixed path's fixed-point scales are
 * reduced over the ranks at load.  The int64 mesh of the mixed path sums
 * exactly (results independent of the rank count).  NCCL (libnccl.so.2) is
 * loaded when first needed.
 *   emu_comm_id: a new communicator id (EMU_COMM_ID_BYTES bytes), made on
 *     one rank and handed to the others by the caller.
 *   emu_attach_comm: joins it (collective over the nranks ranks); must
 *     precede emu_load_particles.  nranks = 1 is allowed.
 * Not available with the adjoint entry points.
 */
#define EMU_COMM_ID_BYTES 128
int emu_comm_id(char* id);
int emu_attach_comm(emu_context* ctx, const char* id, int rank, int nranks);
/*
 * The same sharded schedule with ranks that are contexts of one process, on
 * one GPU or several (no counterpart in the reference): every rank's host
 * thread drives its own context on its own stream, and the library itself
 * does the exchange (a host rendezvous of the ranks at every reduction, then
 * stream-ordered copies and a rank-ordered sum; no kernel waits on another).
 * Used to run the multi-rank path where one GPU is all there is; step
 * graphs are not used by such ranks.
 *   emu_local_group_create: a group of nranks ranks (at most 64).
 *   emu_attach_local: joins rank `rank` of the group (before
 *     emu_load_particles); every rank must then make the same calls in the
 *     same order (loads and steps), each from its own thread.  A rank that
 *     does not arrive within 120 s fails the others' calls (EMU_ERR_STATE).
 *   emu_local_group_destroy: after every member context is destroyed.
 */
int emu_local_group_create(int nranks, void** group);
int emu_attach_local(emu_context* ctx, void* group, int rank);
void emu_local_group_destroy(void* group);

int emu_adjoint_forward(emu_context* ctx, int nsteps, int checkpoint_interval, double start_time, double* dts,
                        emu_run_info* info);
int emu_adjoint_objective(emu_context* ctx, double* J, double* lam_f, double* lam_N);
int emu_adjoint_backward(emu_context* ctx, const double* lam_f_final, const double* lam_N_final, double* lam_f0,
                         double* lam_N0);
int emu_adjoint_reserve(emu_context* ctx, int nsteps, int checkpoint_interval, int64_t* device_bytes,
                        int* stage_store, int* sub_interval);

#ifdef __cplusplus
}
#endif
#endif /* EMU_B200_H_ */
