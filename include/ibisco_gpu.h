/*
 * ibisco_gpu.h — C ABI of the B200 force-and-integrate step for Hybrid IBIsCO.
 *
 * The Fortran host keeps its input/setup phase (main.F90:107-237) and its
 * observables/output (AVERAGE.f90, OUTPUT.F90, WRITETRJ.F90) and replaces the
 * body of its MD loop (NEW_LOOP.F90:66-124, MTS_LOOP.f90:26-44) by calls into
 * this library.  Every entry point is plain C: pointers, sizes and status
 * codes; arrays are passed in the Fortran layout of the reference's MODULE VAR
 * (module_var.F90), column-major with 1-based particle ids.
 *
 * Status codes: 0 on success, a negative IBG_E_* otherwise; the message of the
 * last failure of a context is returned by ibg_last_error().
 */
#ifndef IBISCO_GPU_H
#define IBISCO_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The first group mirrors the reference's fatal STOPs. */
#define IBG_OK 0
#define IBG_E_INVALID (-1)        /* bad argument or descriptor                          */
#define IBG_E_LIST_OVERFLOW (-2)  /* NEW_NEIGHBOUR_WITHLIST.f90:72,113 'LIST TOO SMALL'  */
#define IBG_E_TORSION_TABLE (-3)  /* TORSIONS.inc:105-109 entry not in torsion table     */
#define IBG_E_OOP_RANGE (-4)      /* OUTOFPLANES.inc:62-100 angle outside its table     */
#define IBG_E_FIXED_OVERFLOW (-5) /* a force left the 64-bit fixed-point range           */
#define IBG_E_CELL_GRID (-6)      /* fewer than 3 cells per dimension (MAPS.f90 stencil) */
#define IBG_E_CUDA (-7)           /* CUDA runtime failure                                */
#define IBG_E_TIMEOUT (-8)        /* a bounded device wait ran out                       */
#define IBG_E_TABLE_RANGE (-9)    /* nonbonded distance beyond its table                 */
#define IBG_E_MISSING_TABLE (-10) /* a listed pair has no nonbonded table (INBONDT = 0)   */
#define IBG_E_CAPACITY (-11)      /* device neighbour-list or cell storage exhausted     */
#define IBG_E_IO (-12)            /* input file missing or malformed                     */
#define IBG_E_MEMORY (-13)        /* device memory budget exceeded                       */

/* Precision of the step. */
#define IBG_PREC_FP32_FIXED 0 /* FP32 pair math, 64-bit fixed-point force sums, FP64 integration */
#define IBG_PREC_FP64_PLAIN 1 /* everything in FP64, FP64 atomics (comparison path)             */

/*
 * Descriptor of one system after the reference's setup phase: UNIT, RDCONTROL,
 * ALLOCATEVAR, RDINTERACT, RDCOOR, RDVIRTUAL, MAKE_LISTS, FTABLE, SETLIS,
 * RDVIRTANGLES, BUILD_CONNECTIVITY and RDVIRTBONDS have run.  Field names are
 * the reference's (module_var.F90).  ibg_create deep-copies everything; no
 * pointer is retained after it returns.
 */
typedef struct ibg_desc {
  /* counts */
  int natoms, nvirta, nitems, ntype;
  int numatoms, numbeads, ncoarse;
  /* control (RDCONTROL.f90, ALLOCATEVAR.f90:42-46, main.F90:177-178) */
  int ensemble;   /* 0 NVE, 1 NVT, 2 NPT                                 */
  int nupdate;    /* update_neighbour_list                               */
  int halt_drift; /* halt_drift                                          */
  int nmts;       /* mts; 0 runs the NEW_LOOP body                       */
  int ibrdescr;   /* 0 hybrid (virtual sites present), 1 otherwise       */
  int maxnab;     /* list length at which the reference stops (1000)     */
  float dt, fac, pfac, temp_in, pressure;
  float mktemp, mktemp_atom, mktemp_bead;
  float rcut_atom, rcutsq_atom, rlist_atom;
  float rcut_bead, rcutsq_bead, rlist_bead;
  /* particles */
  const float* mass;       /* MASS(NTYPE)                 */
  const float* invmass;    /* INVMASS(NTYPE)              */
  const int* itype;        /* ITYPE(NITEMS)               */
  const int* type_label;   /* TYPE_LABEL(NITEMS) 1 atom, 2 bead (3 is set for VS on the device) */
  const int* atom;         /* ATOM(NUMATOMS)              */
  const int* bead;         /* BEAD(NCOARSE)               */
  /* topology (SETLIS.f90 output; ld = leading dimension of the 2-D arrays) */
  const int* nbonds;       /* NBONDS(NITEMS)              */
  const int* jbond;        /* JBOND(ld_bond, 4)           */
  int ld_bond;
  const int* nijk;         /* NIJK(NITEMS)                */
  const int* jangleijk;    /* JANGLEIJK(ld_angle, 10)     */
  const int* kangleijk;
  int ld_angle;
  const int* nijkl;        /* NIJKL(NITEMS)               */
  const int* jtorijkl;     /* JTORIJKL(ld_torsion, 10)    */
  const int* ktorijkl;
  const int* ltorijkl;
  int ld_torsion;
  const int* noopijkl;     /* NOOPIJKL(NITEMS)            */
  const int* joopijkl;     /* JOOPIJKL(ld_oop, 20)        */
  const int* koopijkl;
  const int* loopijkl;
  int ld_oop;
  /* exclusions (BUILD_CONNECTIVITY.f90, RDVIRTBONDS.f90) */
  const int* connections;  /* CONNECTIONS(NITEMS)         */
  const int* connected_to; /* CONNECTED_TO(ld_conn, 20)   */
  int ld_conn;
  /* type maps, dense, first index fastest */
  const int* ibondt;  /* IBONDT(NTYPE,NTYPE)             */
  const int* inbondt; /* INBONDT(NTYPE,NTYPE)            */
  const int* iangt;   /* IANGT(NTYPE,NTYPE,NTYPE)        */
  const int* itort;   /* ITORT(NTYPE,NTYPE,NTYPE,NTYPE)  */
  const int* ioopt;   /* IOOPT(NTYPE,NTYPE,NTYPE,NTYPE)  */
  const int* bond_type_label;    /* (NBTYPE) 1 atomistic, 2 CG, 3 mixed */
  const int* angle_type_label;   /* (NATYPE)  */
  const int* torsion_type_label; /* (NTTYPE)  */
  const int* oop_type_label;     /* (NOTYPE)  */
  /* tables after FTABLE.f90.  Bonded tables are X(NTYPES, 0:ld-1), type fastest;
     the nonbonded tables are X(0:ld_nb-1, NNBTYPE), index fastest, as in the
     reference (ld = MAXINPUT+1 there). */
  int nbtype, natype, nttype, nnbtype, notype;
  int ld_b, ld_a, ld_t, ld_nb, ld_o;
  const int* ndatb;  const float* binb;  const float* rbond;     const float* bond_pot; const float* bond_force;
  const int* ndatan; const float* bina;  const float* angle;     const float* bend_pot; const float* bend_force;
  const int* ndatt;  const float* bint;  const float* angle_tor; const float* tor_pot;  const float* tor_force;
  const int* ndatnb; const float* binnb; const float* rnbond;    const float* nbond_pot; const float* nbond_force;
  const int* ndato;  const float* bino;  const float* angle_oop; const float* oop_pot;  const float* oop_force;
  /* virtual sites (RDVIRTUAL.f90) */
  int ld_vs, vs_maxatoms;
  const int* vitype;          /* VITYPE(NVIRTA)                        */
  const int* virt_center;     /* VIRT_CENTER(NVIRTA), 0 = centre of mass */
  const int* virt_numatoms;   /* VIRT_NUMATOMS(NTYPE)                  */
  const int* virt_atm_ind;    /* VIRT_ATM_IND(ld_vs, vs_maxatoms)      */
  const float* virt_invmass;  /* VIRT_INVMASS(NTYPE)                   */
  const float* virt_masscoeff;/* VIRT_MASSCOEFF(NTYPE,NTYPE)           */
} ibg_desc;

/* Per-step observables: what AVERAGE.f90, OUTPUT.F90 and WRITETRJ.F90 read. */
typedef struct ibg_obs {
  double ek[2];          /* EK(1) atoms, EK(2) beads                         */
  double temp, temp_atom, temp_bead;
  double v_nb[3], v_bond[3], v_angle[3], v_torsion[3], v_oop[3];
  double pt[6];          /* PT11, PT22, PT33, PT12, PT13, PT23 (after /V)    */
  double box[3];
  long long bond_overext;/* BONDS.inc:21-28 warnings this step               */
  long long cell_clamps; /* coordinates at +L/2 folded into the last cell    */
  int step, status;
} ibg_obs;

typedef struct ibg_ctx ibg_ctx;
typedef struct ibg_setup ibg_setup;

/* ---------------------------------------------------------------- setup --
 * Host-side setup from a directory of reference input files (control,
 * interaction and its tables, coordinate, virtual, virtbonds, virtangles).
 * Replaces main.F90:107-218 for hosts that are not the Fortran program; the
 * descriptor it yields is what a Fortran host fills from MODULE VAR.
 * initial_state receives SXYZ(3,NATOMS), VXYZ(3,NATOMS) (reduced units) and BOX.
 */
int ibg_setup_read(const char* dir, ibg_setup** out, char* err, int errlen);
/* The same reader chain on input files held in memory: nfiles buffers, each
   with the file name the control and interaction files refer to ("control",
   "interaction", "coordinate", "virtual", "virtbonds", "virtangles" and every
   table file), data[k] of sizes[k] bytes.  A host that builds its inputs in
   memory, such as an iterative Boltzmann inversion loop writing new trial
   potentials, sets systems up without touching the file system
   (RDINTERACT.f90, RDCOOR.f90 and RDVIRTUAL.f90 read those files). */
int ibg_setup_read_mem(int nfiles, const char* const* names, const char* const* data, const long* sizes,
                       ibg_setup** out, char* err, int errlen);
/* Replace nonbonded table `table` (1..NNBTYPE) of a setup by nrows rows
   r(nm), V(kJ/mol): the two columns of a table file, as REAL*4.  The rows go
   through RDINTERACT.f90:504-533 (unit conversion, a row at r = 0 inserted
   when r(1) is not 0) and FTABLE.f90:59-75, exactly as a file with those values
   would; the setup's descriptor points to the new tables afterwards.  The
   interaction of an IBI iteration changes its potentials this way between
   trial runs. */
int ibg_setup_set_nb_table(ibg_setup* s, int table, int nrows, const float* r, const float* v);
const ibg_desc* ibg_setup_desc(const ibg_setup* s);
int ibg_setup_initial_state(const ibg_setup* s, float* sxyz, float* vxyz, float* box);
/* Integer/float scalars of the control file not carried by the descriptor:
   [0] num_of_time_steps [1] trajectory [2] initialize_velocities (1 = Y). */
int ibg_setup_control(const ibg_setup* s, int* ivals, int n);
/* Named array of the setup (e.g. "CONNECTED_TO", "BOND_FORCE"); returns its
   length, or -1 when the name is unknown.  out may be NULL to query. */
long ibg_setup_array_i(const ibg_setup* s, const char* name, int* out, long n);
long ibg_setup_array_f(const ibg_setup* s, const char* name, float* out, long n);
void ibg_setup_free(ibg_setup* s);

/* --------------------------------------------------------------- device --
 * ibg_create: copies the descriptor to the current CUDA device.
 * ibg_set_state: positions SXYZ(3,NATOMS) (unwrapped), velocities
 *   VXYZ(3,NATOMS), box(3); then runs the reference's pre-loop
 *   initialisation (main.F90:150-234: virtual sites, SHIFT, initial
 *   temperatures, cell maps, first Verlet lists).
 * ibg_step: one loop body (NEW_LOOP.F90:66-124 or MTS_LOOP.f90:26-44) for
 *   step number `step`; `out` (may be NULL) receives the observables.
 * ibg_forces: the same body up to and including the force stage, without
 *   MOVE/MOMENTUM/SCALEBP (for force parity checks).
 * ibg_run: steps first..first+nsteps-1 with CUDA-graph replay; per_step (may
 *   be NULL) receives nsteps observables.
 * ibg_get_state: SXYZ/RXYZ/FXYZ (3,NITEMS) and VXYZ (3,NATOMS) as REAL*4;
 *   any pointer may be NULL.  ibg_get_state_f64: the FP64 state.
 * ibg_get_neighbour_list: LIST(maxnab,N) of list `which` (0 atoms, 1 beads)
 *   in the reference's order, 1-based global ids, 0-terminated, and
 *   NNEBS(INDEX_LIST(A)) for A=1..N; list or nnebs may be NULL.
 * ibg_get_exclusions: CONNECTIONS(NITEMS) and CONNECTED_TO(NITEMS,20) as held
 *   on the device.
 */
int ibg_create(const ibg_desc* d, int precision, ibg_ctx** out);
int ibg_set_state(ibg_ctx* c, const float* sxyz, const float* vxyz, const float* box);
int ibg_step(ibg_ctx* c, int step, ibg_obs* out);
int ibg_forces(ibg_ctx* c, int step, ibg_obs* out);
int ibg_run(ibg_ctx* c, int first_step, int nsteps, ibg_obs* per_step);
int ibg_get_state(ibg_ctx* c, float* sxyz, float* rxyz, float* vxyz, float* fxyz);
int ibg_get_state_f64(ibg_ctx* c, double* sxyz, double* vxyz, double* fxyz);
int ibg_get_neighbour_list(ibg_ctx* c, int which, int* list, int maxnab, int* nnebs);
int ibg_get_exclusions(ibg_ctx* c, int* connections, int* connected_to);
/* Device-side timing with CUDA events on the context's stream.
   stage_ms[5] = milliseconds of the last ibg_run/ibg_step call (always).
   With timing on (ibg_set_timing(c,1): direct launches, no graph replay),
   stage_ms[0..4] accumulate the time of the list build, nonbonded, bonded,
   integration/reduction and remaining kernels since ibg_set_timing, and
   stage_ms[6] counts the nonbonded launches, stage_ms[8] those of them that
   ran the bead list; stage_ms[7] counts the growths of the Verlet-list
   storage (nstage <= 9).  launches = kernels enqueued by this context so
   far. */
int ibg_set_timing(ibg_ctx* c, int on);
int ibg_get_timing(ibg_ctx* c, double* stage_ms, int nstage, long long* launches);
/* Benchmark support: before every step of ibg_run write `bytes` of scratch
   memory (evicting the L2 cache) and time only the steps (stage_ms[5]). */
int ibg_set_l2_flush(ibg_ctx* c, long long bytes);
/* Diagnostic: replace the Verlet-list storage by `rows` rows of 32 entries per
   slice.  The stored lists are discarded, so call it only right before a step
   that rebuilds them (step % update_neighbour_list == 0); a build that does not
   fit stops the run at that step, the storage grows and the step is repeated
   (the same path a growing system takes).  stage_ms[7] of ibg_get_timing
   counts the growths. */
int ibg_set_list_rows(ibg_ctx* c, int rows);
/* Form of the stored Verlet lists (FP32 path; the FP64 path always keeps
   IBG_LIST_PER_PARTICLE).  IBG_LIST_PER_PARTICLE: a list per particle, eight
   lanes of the nonbonded kernel per particle.  IBG_LIST_PER_SLICE: a list per
   slice of four consecutive slots holding each neighbour once, with a mask of
   which of the four it pairs with.  Both hold the reference's half-list
   pairs, so ibg_get_neighbour_list returns the same LIST and NNEBS and every
   force sum is bit for bit the same; the slice form gathers each stored
   neighbour's position and adds its force once per slice.  On the
   2,000,000-bead melt that cuts the nonbonded kernel's DRAM traffic from
   1.06 GB to 0.45 GB a launch and its time by 3 %; its list build is slower,
   and with lists rebuilt every 10 steps a step takes 1.656 ms against
   1.669 ms (0.0887 against 0.0941 ms on a 40,000-bead melt).  IBG_LIST_AUTO
   (the default): slice lists for lists of at least 2*64*32 particles per SM
   of the device (606,208 on 148 SMs), per-particle lists below.  Changing
   the form discards the stored lists: ibg_set_state must be called again
   before the next step.  ibg_get_list_form returns the form in use (of the
   atom list, or of the bead list when there is no atom list):
   IBG_LIST_PER_PARTICLE or IBG_LIST_PER_SLICE. */
#define IBG_LIST_AUTO (-1)
#define IBG_LIST_PER_PARTICLE 0
#define IBG_LIST_PER_SLICE 1
int ibg_set_list_form(ibg_ctx* c, int form);
int ibg_get_list_form(const ibg_ctx* c);
/* Launch tuning of the nonbonded kernel: nb_tables_smem stages the tables in
   shared memory per block (1) or reads them through L1 (0; the FP32 default,
   the FP64 path stages them); nb_blocks_per_sm limits the resident blocks per
   SM (0: all that fit); nb_chunk (FP32 path): each block works through its
   own contiguous range of work units (neighbouring slices), so its warps
   gather from one region of space, and the last nb_chunk/256 of the units are
   taken dynamically by whichever warps finish first (0: every warp takes
   units alone, dynamically); nb_rows: list rows per work unit, 8 or 16 (0:
   16); nb_window (FP32 path, nb_chunk > 0): 0 gives each block one contiguous
   range of units, W > 0 deals runs of W consecutive units to the blocks in
   turn, so that all blocks work through one region of space at a time.  Forces and trajectories do not depend on the tuning (integer force
   sums); on the FP32 path nonbonded energies and virials are summed in groups
   of 8 list rows before their exact fixed-point sum, so they do not depend on
   it either.  Set it before a batch is made of the context.
   ibg_autotune: times each candidate tuning on the context's current lists
   (reps launches each, CUDA events; with an L2 flush set by ibg_set_l2_flush,
   each launch starts from a flushed L2, as a timed step does), keeps the
   fastest, writes it to best, and candidate k and its microseconds per launch
   to cand[k] and us[k] (k < ncand; either may be NULL); returns the number of
   candidates.  It leaves the system's state unchanged. */
typedef struct ibg_tuning {
  int nb_tables_smem;
  int nb_blocks_per_sm;
  int nb_chunk;
  int nb_rows;
  int nb_window;
} ibg_tuning;
int ibg_get_tuning(const ibg_ctx* c, ibg_tuning* t);
int ibg_set_tuning(ibg_ctx* c, const ibg_tuning* t);
int ibg_autotune(ibg_ctx* c, int reps, ibg_tuning* best, ibg_tuning* cand, double* us, int ncand);
/* Centre-of-mass virtual sites (VIRT_CENTER = 0).  VIRTUAL_DEF.f90:30-39 sums
   MASS*SXYZ over a site's members, but before each site resets only the x
   component of its sum (VIRTUAL_DEF.f90:31); the y and z sums run on from one
   such site to the next within a pass.  IBG_VS_COM_FIXED (the default)
   resets all three, giving each site its centre of mass; IBG_VS_COM_REFERENCE
   reproduces the reference's running y and z sums (one warp walks the sites
   in order, so it is slow on many sites).  Centre-atom sites are the same in
   both.  Set it before ibg_set_state and before a batch is made of the
   context. */
#define IBG_VS_COM_FIXED 0
#define IBG_VS_COM_REFERENCE 1
int ibg_set_vsite_com(ibg_ctx* c, int form);
/* Device memory a context holds (bytes), and an estimate made before creating
   one from its descriptor and box; the estimate includes the Verlet-list
   storage the first list build will need, with margin.  A serving loop admits
   systems by these figures. */
long long ibg_device_bytes(const ibg_ctx* c);
long long ibg_estimate_bytes(const ibg_desc* d, int precision, const float* box);
/* Select the CUDA device of the calling thread for subsequent ibg_create. */
int ibg_set_device(int device);
const char* ibg_last_error(const ibg_ctx* c);
void ibg_destroy(ibg_ctx* c);

/* Library version string. */
const char* ibg_version(void);

/* --------------------------------------------------------------- output --
 * The trajectory and restart files of WRITETRJ.F90, for hosts that are not the
 * Fortran program (the Fortran host keeps its own WRITETRJ).  A host runs
 * NTRJ steps with ibg_run, reads the state with ibg_get_state and writes:
 * ibg_trz_write: one TRZ frame after step `step` (WRITETRJ.F90:28-97): Fortran
 *   unformatted sequential records with 4-byte length markers, as gfortran
 *   writes them; the title and record count precede the first frame; obs of
 *   that step (box, pressure tensor, energies), SXYZ(3,NATOMS) and
 *   VXYZ(3,NATOMS) in reduced units as ibg_get_state returns them.
 * ibg_write_restart: the restart file in the coordinate file's format
 *   (WRITETRJ.F90:119-178): positions as G21.14, velocities as F16.10 nm/ps,
 *   the setup's molecules, types and bonds; RDCOOR.f90 reads it back. */
typedef struct ibg_trz ibg_trz;
int ibg_trz_open(const ibg_setup* s, const char* path, ibg_trz** out);
int ibg_trz_write(ibg_trz* t, int step, const ibg_obs* obs, const float* sxyz, const float* vxyz);
void ibg_trz_close(ibg_trz* t);
int ibg_write_restart(const ibg_setup* s, const char* path, int step, const float* box, const float* sxyz,
                      const float* vxyz);

/* ---------------------------------------------------------------- batch --
 * Many independent systems stepped together on one GPU.  A batch packs its
 * systems into one kernel launch per stage (blocks are mapped to systems) and
 * replays the whole batch step as one CUDA graph.  This is the form in which
 * many small or mid-size systems, such as iterative Boltzmann inversion trial
 * runs each with its own tables, fill the GPU.  Every system keeps its own
 * step counter, list schedule, MTS phase, thermostat and barostat, and its
 * results are bitwise the same as when it runs alone.
 *
 * ibg_batch_create: contexts of one device and precision, each after
 *   ibg_set_state and in no other batch.  The batch refers to the contexts;
 *   destroy it before any of them.  Contexts stay usable on their own between
 *   batch runs (ibg_run, ibg_get_state, ...).
 * ibg_batch_run: advances every system by nsteps steps from its own last step
 *   (the step of its last ibg_run/ibg_step or batch run; 0 after
 *   ibg_set_state), or only up to last_step[s] when last_step is given.
 *   last_obs (may be NULL) receives, per system, the observables of the last
 *   step it ran.
 * ibg_batch_get_timing: device milliseconds of the last ibg_batch_run (CUDA
 *   events on the batch's stream) and kernels launched by the batch so far. */
typedef struct ibg_batch ibg_batch;
int ibg_batch_create(ibg_ctx* const* ctxs, int n, ibg_batch** out);
int ibg_batch_run(ibg_batch* b, int nsteps, const int* last_step, ibg_obs* last_obs);
int ibg_batch_size(const ibg_batch* b);
int ibg_batch_get_timing(const ibg_batch* b, double* run_ms, long long* launches);
const char* ibg_batch_last_error(const ibg_batch* b);
void ibg_batch_destroy(ibg_batch* b);

/* ---------------------------------------------------- no-allocation path --
 * ibg_nonbonded_static: the nonbonded forces, energies and virial of one
 * particle list, for callers that cannot allocate device memory at the time
 * they need them (a host whose device memory all belongs to its own
 * allocator, a loop that must not let cudaMalloc/cudaFree synchronise the
 * device).  It has no counterpart in the reference: it is NONBONDED_FORCE on
 * the reference's own arrays, offered without a context.  Every pointer
 * except box, err and stream is device memory owned by the caller, in the
 * reference's layout and 1-based ids: rxyz(3,nitems) wrapped positions,
 * itype/type_label(nitems) (3 for virtual sites), index_list(n),
 * list(maxnab,n), nnebs(nitems), inbondt(ntype,ntype),
 * rnbond/nbond_force/nbond_pot(ld_nb,nnbtype), binnb/ndatnb(nnbtype).
 * Outputs: fxyz(3,nitems) in FP64 (the forces of this list alone) and sums[9]
 * = V_NB(1..3), PT11, PT22, PT33, PT12, PT13, PT23 (not divided by the volume).
 * Scratch is a fixed __device__ array in the library, sized for
 * IBG_STATIC_MAX_PARTICLES particles; larger inputs return IBG_E_CAPACITY.
 * The first call on a device looks up that array's address with the device
 * current, so make it before any stream capture.  All calls share the array:
 * calls that overlap on the GPU (other streams, other host threads) race.
 * The call waits for `stream` (a cudaStream_t, may be NULL) before it returns,
 * to read its error word, and allocates nothing.  ntype, nnbtype >= 1 and
 * ld_nb >= 2 (IBG_E_INVALID otherwise); a particle type outside 1..ntype or an
 * INBONDT entry outside 1..nnbtype on a pair inside the cutoff returns
 * IBG_E_MISSING_TABLE, a table row whose successor lies beyond ld_nb or beyond
 * NDATNB+1 IBG_E_TABLE_RANGE, an id outside 1..nitems in index_list or list
 * IBG_E_INVALID.  err (may be NULL) receives a message. */
#define IBG_STATIC_MAX_PARTICLES 262144
#define IBG_STATIC_MAX_BLOCKS 1024
int ibg_nonbonded_static(int nitems, int n, const float* rxyz, const int* itype, const int* type_label,
                         const int* index_list, const int* list, int maxnab, const int* nnebs, int ntype,
                         const int* inbondt, int nnbtype, int ld_nb, const float* rnbond,
                         const float* nbond_force, const float* nbond_pot, const float* binnb,
                         const int* ndatnb, const float* box, float rcutsq, double* fxyz, double* sums,
                         void* stream, char* err, int errlen);

/* -------------------------------------------------------------- serving --
 * A service of simulation jobs on one GPU with continuous batching.  Jobs are
 * submitted from any host thread; one service thread admits them in order
 * while the job-slot count and the device-memory budget allow (estimated with
 * ibg_estimate_bytes, accounted with ibg_device_bytes), keeps their state,
 * lists and tables resident, steps all admitted jobs together as one batch,
 * tick_steps steps per tick, each up to its own step count, and retires
 * finished jobs between ticks (final state to host memory, device memory
 * freed).  Jobs that arrive while others run join at the next tick.  A job's
 * result is bitwise the same as the same system run alone with ibg_run.
 *
 * ibg_server_create: hbm_budget <= 0 takes 80 % of the free device memory.
 * ibg_server_submit: the server takes ownership of the setup (it frees it) and
 *   runs steps 1..nsteps from the setup's initial state.
 * ibg_server_wait: blocks until the job is done or failed (timeout_s < 0: no
 *   limit) and returns its state (IBG_JOB_*).
 * ibg_server_result: SXYZ(3,NITEMS) and VXYZ(3,NATOMS) after the last step,
 *   its observables, and times[3] = seconds queued, seconds from admission to
 *   completion, latency (submission to completion); any pointer may be NULL.
 * ibg_server_get_stats: counts, latency percentiles over completed jobs, jobs/s and
 *   atom-steps/s over the span from the first submission to the last
 *   completion, GPU time of the ticks, and peak residency. */
#define IBG_JOB_QUEUED 0
#define IBG_JOB_RUNNING 1
#define IBG_JOB_DONE 2
#define IBG_JOB_FAILED 3
typedef struct ibg_server ibg_server;
typedef struct ibg_server_stats {
  long long submitted, done, failed, running, queued;
  double p50_s, p99_s, mean_s, span_s, jobs_per_s;
  long long atom_steps;
  double atom_steps_per_s, gpu_s;
  long long ticks, batch_builds;
  long long peak_jobs, peak_bytes, budget_bytes;
} ibg_server_stats;
int ibg_server_create(int device, int precision, long long hbm_budget, int max_jobs, int tick_steps,
                      ibg_server** out);
int ibg_server_submit(ibg_server* s, ibg_setup* setup, int nsteps, long long* job);
int ibg_server_wait(ibg_server* s, long long job, double timeout_s);
int ibg_server_drain(ibg_server* s, double timeout_s);
int ibg_server_result(ibg_server* s, long long job, float* sxyz, float* vxyz, ibg_obs* last_obs, double* times);
const char* ibg_server_job_error(ibg_server* s, long long job);
int ibg_server_get_stats(ibg_server* s, ibg_server_stats* out);
void ibg_server_destroy(ibg_server* s);

#ifdef __cplusplus
}
#endif
#endif /* IBISCO_GPU_H */
