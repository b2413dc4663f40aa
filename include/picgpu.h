/*
 * picgpu.h -- C-ABI of the B200 IFE-PIC step library (libpicgpu.so).
 *
 * Every entry point is plain C: pointers, sizes, return codes.  No torch or
 * CUDA types cross this boundary, so a Fortran main program binds it with
 * ISO_C_BINDING interface blocks and Python binds it with ctypes.
 *
 * Each entry point names the reference subroutine it replaces.  Paths are
 * relative to the PIC-IFE_GEC project of weqwoueu/pic-.
 *
 * Conventions
 *  - Node n of an nnx x nny uniform mesh is n = i*nny + j (0-based i, j);
 *    its Fortran id is n+1 = (i-1)*nny + j with 1-based i, j
 *    (code/IFE-Rectangular/Cubic_Partition_2D.f90:60-66).
 *  - Element e = i*(nny-1) + j; Fortran id e+1 = j + (i-1)*(nny-1); corners
 *    HT(1:4,e) = (i,j), (i+1,j), (i+1,j+1), (i,j+1)
 *    (code/IFE-Rectangular/Cubic_Partition_2D.f90:70-90).
 *  - Index tables handed to pic_init (CSR rows/columns, patches) are 1-based
 *    like the Fortran arrays they mirror; they are converted once at init.
 *  - Return value 0 = ok, negative = error class (PIC_ERR_*).  Details of
 *    the last failure are in pic_last_error().  Nothing calls exit/abort.
 *  - Not re-entrant: one context per process, one CUDA device, one stream.
 */
#ifndef PICGPU_H
#define PICGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PIC_OK 0
#define PIC_ERR_ARG (-1)        /* bad argument or size                 */
#define PIC_ERR_CUDA (-2)       /* CUDA runtime / launch failure        */
#define PIC_ERR_SOLVER_CAP (-3) /* PCG reached its iteration cap        */
#define PIC_ERR_NAN (-4)        /* NaN/Inf in a field or residual       */
#define PIC_ERR_DOMAIN (-5)     /* particle outside the mesh            */
#define PIC_ERR_STATE (-6)      /* call out of order (no init, ...)     */
#define PIC_ERR_CAPACITY (-7)   /* particle array capacity exceeded     */
#define PIC_ERR_SETUP (-8)      /* geometry the mesh builder rejects    */
#define PIC_ERR_BREAKDOWN (-9)  /* PCG breakdown (rho or p.Ap == 0)     */

#define PIC_MAX_SPECIES 4
#define PIC_MAX_OBJECTS 32
#define PIC_MAX_REACTIONS 8

/* Object shapes, same codes as objects(i)%Shape in INPUT/object.inp. */
#define PIC_SHAPE_CIRCLE 1
#define PIC_SHAPE_BOX 3
#define PIC_SHAPE_ELLIPSE 5

/* Wall treatment of particles (MCC_jw/code/Interface_IFE/MCCInterface.f90:361-532). */
#define PIC_WALL_ABSORB 0
#define PIC_WALL_REFLECT 1

/* Arithmetic of the step. */
#define PIC_PREC_FP64 0  /* plain FP64 path                                  */
#define PIC_PREC_MIXED 1 /* FP32 cell-relative push, FP32 PCG in FP64 refine */

/* Linear solver of pic_ife_solve. */
#define PIC_SOLVER_JPCG 0 /* Jacobi-PCG, MY_PCG.f90                   */
#define PIC_SOLVER_FCG_UNET 1 /* flexible CG with the learned preconditioner */

typedef struct pic_object {
  int32_t shape;     /* PIC_SHAPE_*                                          */
  int32_t conductor; /* 1: nodes inside are Dirichlet at phi                 */
  double cx, cy;     /* centre (circle/ellipse) or lower-left corner (box)   */
  double a, b;       /* radius (a); ellipse semi-axes; box upper-right (a,b) */
  double angle;      /* ellipse rotation (rad)                               */
  double eps;        /* relative permittivity inside (objects(i)%Eps)        */
  double phi;        /* normalised potential of a conductor                  */
} pic_object;

/* Deck for the host-side mesh builder (Setup_IFE_Mesh_2D + IFE_Start_2D +
 * Get_PointPatch).  Lengths and potentials are normalised (L_ref, Phi_ref). */
typedef struct pic_deck {
  int32_t nnx, nny;            /* nodes per direction                        */
  double xmin, xmax, ymin, ymax;
  int32_t delta;               /* 0 Cartesian; 1 axisymmetric r-z (x = z,
                                  y = r, the axis at y = ymin = 0); pic_init
                                  takes delta 1 with PIC_PREC_FP64 only       */
  int32_t wall_dirichlet[4];   /* left, right, bottom, top: 1 Dirichlet       */
  double wall_phi[4];          /* Dirichlet values                            */
  int32_t n_objects;
  pic_object objects[PIC_MAX_OBJECTS];
} pic_deck;

/* Arrays the reference holds after its setup phase (IFE_Data module). */
typedef struct pic_mesh_desc {
  int32_t nnx, nny;
  double xmin, xmax, ymin, ymax;
  int32_t delta;
  const int32_t *node_type;     /* [nodes] node_type(2,:): >0 unknown id, <0 Dirichlet */
  const int32_t *node_index;    /* [nodes] -1 outside objects, object region (<=-2) inside */
  const int32_t *element_index; /* [elems] -1 outside, <=-2 inside object, >0 interface id */
  const double *phi_dirichlet;  /* [nodes] potential on Dirichlet nodes          */
  const double *cell_volume;    /* [nodes] Cell_Volume_zwz(2,:)                  */
  int32_t n_unknowns;
  int64_t nnz;
  const int32_t *a_srow;   /* [n_unknowns+1] 1-based (SPARSE%SROW of A_stiff)   */
  const int32_t *a_jcol;   /* [nnz] 1-based unknown ids (SPARSE%JCOL)           */
  const double *a_k;       /* [nnz] (SPARSE%K)                                  */
  int64_t nnz_xt;
  const int32_t *xt_srow;  /* [n_unknowns+1] A_stiff_xt rows                    */
  const int32_t *xt_jcol;  /* [nnz_xt] 1-based NODE ids of Dirichlet columns    */
  const double *xt_k;
  const double *a_diag;    /* [n_unknowns] Jacobi diagonal A_diag               */
  const double *rhs_fix;   /* [n_unknowns] rhs_FIX (Neumann), may be NULL       */
  const double *mass_q1;   /* [16] Q1 element load matrix, row j col k          */
  int32_t n_interface;
  const double *ife_mass;  /* [n_interface*16] interface-element load matrices  */
  const int32_t *patch_ptr;   /* [nodes+1] 0-based offsets into patch_nodes      */
  const int32_t *patch_nodes; /* 1-based node ids (point_patch(i,2:))             */
  int32_t n_objects;
  const pic_object *objects;
  const double *mass_rows; /* delta 1: [ (nny-1) * 16 ] r-weighted Q1 load matrix
                              of each element row, row-major; NULL for delta 0 */
} pic_mesh_desc;

typedef struct pic_species_desc {
  double charge;      /* qs, units of e                                      */
  double mass;        /* kg                                                  */
  double weight;      /* real particles per macro-particle (ParticleBundle%Weight) */
  int64_t capacity;   /* particle slots to reserve in HBM                    */
} pic_species_desc;

typedef struct pic_params {
  int32_t n_species;
  pic_species_desc species[PIC_MAX_SPECIES];
  double dt;          /* normalised time step                                */
  double n_ref;       /* m^-3                                                */
  double T_ref_eV;    /* eV                                                  */
  double pcg_tol;     /* relative residual ||r||/||b|| (PCG_Tol)             */
  int32_t pcg_maxit;  /* PCG_MaxIT                                           */
  int32_t wall_bc[4]; /* particle treatment at left, right, bottom, top      */
  uint64_t seed;      /* Philox key                                          */
  int32_t precision;  /* PIC_PREC_*                                          */
  int32_t sort_interval; /* counting sort every k steps in pic_step (>=1)    */
  int32_t solver;     /* PIC_SOLVER_*                                        */
  int32_t diag_interval; /* pic_step deposits the per-node energy (Ek_tot, a
                          * diagnostic) on steps that are multiples of this;
                          * <= 1: every step.  pic_get_par_chg always does. */
} pic_params;

/* One MCC_jw collision bundle (Type MCCBundle, mc/TypeMCC.f90:9-20). */
typedef struct pic_mcc_table {
  int32_t species;       /* colliding species                                */
  int32_t n_reaction;
  int32_t n_sigma;
  double energy_min;     /* log10(eV) of the first grid point                */
  double energy_interval;/* log10 step                                       */
  double energy_max;     /* eV of the last grid point                        */
  double collision_ratio;/* P_null = 1 - exp(-nu_max dt)                     */
  int32_t reaction_type[PIC_MAX_REACTIONS]; /* 11,12,13 (e-) or 101,103 (ion) */
  double threshold[PIC_MAX_REACTIONS];      /* eV                              */
  int32_t resultant[PIC_MAX_REACTIONS];     /* species created (ionisation)    */
  const double *probability; /* [n_sigma*n_reaction] cumulative, normalised  */
} pic_mcc_table;

typedef struct pic_gas {
  double mass;        /* kg                                                   */
  double temperature; /* K                                                    */
  double density;     /* m^-3                                                 */
} pic_gas;

typedef struct pic_solve_stats {
  int32_t iterations;     /* PCG iterations performed                        */
  int32_t ierr;           /* MY_PCG IERR: 0 ok, 1 cap, 2 rho0==0, 3 p.Ap==0   */
  double rel_residual;    /* sqrt(normR/normRHS) at exit                      */
  double ms;              /* device time of the solve                         */
  int32_t fallback;       /* 0, or why flexible CG handed over to Jacobi-PCG:
                           * 1 cap, 2 breakdown (p.Ap <= 0), 3 stall, 4 NaN,
                           * 5 preconditioner failed, 6 true residual above
                           * tolerance after restarts                         */
  int32_t outer;          /* FP64 refinement sweeps (mixed precision)         */
} pic_solve_stats;

typedef struct pic_mcc_stats {
  int64_t n_selected[PIC_MAX_SPECIES];
  int64_t n_by_reaction[PIC_MAX_SPECIES][PIC_MAX_REACTIONS];
  int64_t n_created[PIC_MAX_SPECIES];
} pic_mcc_stats;

typedef struct pic_step_stats {
  int64_t n_particles[PIC_MAX_SPECIES]; /* live after the step                */
  int64_t n_lost[PIC_MAX_SPECIES];      /* absorbed this step                 */
  pic_solve_stats solve;
  pic_mcc_stats mcc;
  double ms_push, ms_solve, ms_ppr, ms_mcc, ms_sort, ms_total;
  double ms_push_kernel;  /* device time of the fused push kernels alone      */
  int64_t pushed;         /* particles pushed (live at the start of the step) */
} pic_step_stats;

/* ---- mesh builder (host C++; replaces the reference's setup chain) ---- */

/* Builds the arrays of pic_mesh_desc from a deck:
 *   Partition_Cube_2D.f90 (node_type), Cubic_Partition_2D.f90 (HP/HT),
 *   El_Object_Intersection_info_2D_BL.f90 (interface elements),
 *   Generate_stiffness_matrix_local_IFE.f90 + IFE_Start_2D.f90:320-479 (CSR),
 *   Global_RHS_PDE_2D.f90 / IFE_RHS_2D.f90 (load matrices),
 *   SetupGrids_2D_QLL.f90:197-330 (Cell_Volume_zwz), Get_PointPatch.f90.
 * On success *out points at storage owned by the library until
 * pic_mesh_free(*out). */
int pic_mesh_build(const pic_deck *deck, pic_mesh_desc **out);
/* The same descriptor, with the interface elements' Q1 IFE basis, element
 * stiffness and load matrices (Retangular_reference_basis_IFE.f90,
 * Gauss_integration_local_stiffness_IFE.f90, IFE_RHS_2D.f90) computed in
 * FP64 on the current CUDA device, one thread per interface element, by the
 * same code the host builder runs: the result equals pic_mesh_build's bit
 * for bit.  Allocates and frees its own device scratch; PIC_ERR_CUDA if no
 * device is usable. */
int pic_mesh_build_device(const pic_deck *deck, pic_mesh_desc **out);
void pic_mesh_free(pic_mesh_desc *mesh);
/* Interface-element geometry for diagnostics/tests: per interface element
 * (1-based id k) the element number, type (1 corner cut, 2 opposite edges),
 * reference-vertex map pointer_reference_to_local(1:4), beta1, beta2, D, E. */
int pic_mesh_interface_info(const pic_mesh_desc *mesh, int32_t k, int32_t *element,
                            int32_t *type, int32_t *ref_to_local, double *beta,
                            double *d, double *e);
/* Q1 IFE basis of interface element k (Retangular_local_basis_IFE.f90):
 * value and gradient of local basis `basis` (0..3, HT order) at (x, y). */
int pic_mesh_ife_basis(const pic_mesh_desc *mesh, int32_t k, int32_t basis, double x,
                       double y, double *value, double *dx, double *dy);

/* ---- device context ---- */

/* pic_init: copies the mesh tables to HBM, splits the stiffness into the
 * regular Q1 stencil and explicit interface/boundary rows, builds the PPR
 * pseudo-inverse rows, allocates particle storage.  Replaces the module
 * state set up before Main_IFE_Test_2.f90:278. */
int pic_init(const pic_mesh_desc *mesh, const pic_params *params);
void pic_finalize(void);
const char *pic_last_error(void);

/* MCC_jw tables (MCCInit.F90:29-152) and gas, one table per colliding species. */
int pic_mcc_init(const pic_gas *gas, int32_t n_tables, const pic_mcc_table *tables);

/* Particle bundle I/O (ParticleBundle%Dump/Load, ParticleBundle.f90:286-375).
 * id may be NULL (ids 0..n-1 are assigned); loc may be NULL (located on upload). */
int pic_upload_particles(int32_t species, int64_t n, const double *x, const double *y,
                         const double *vx, const double *vy, const double *vz,
                         const int32_t *loc, const uint32_t *id);
/* Copies the live particles in device order.  Any output pointer may be NULL. */
int pic_download_particles(int32_t species, int64_t capacity, double *x, double *y,
                           double *vx, double *vy, double *vz, int32_t *loc,
                           uint32_t *id, int64_t *n_out);
int pic_particle_count(int32_t species, int64_t *n);
/* The id the next particle created in `species` (MCC ionisation) receives.
 * pic_upload_particles sets it to the largest uploaded id + 1; a restart
 * restores the saved value with pic_set_next_id, which refuses values below
 * the current one (ids would repeat).  Created particles draw their random
 * numbers by id, so a restart that kept a smaller next id would diverge.
 * The reference keeps no particle ids (ParticleBundle.f90:286-375 dumps the
 * particles without them). */
int pic_get_next_id(int32_t species, uint32_t *next_id);
int pic_set_next_id(int32_t species, uint32_t next_id);

/* ParticlePositioning / InjectPositioning (ParticlePositioning.f90,
 * InjectPositioning.f90:1-24, call site GetParChg_2D.f90:137-163):
 * element of every particle of `species` (-1 for all species). */
int pic_particle_positioning(int32_t species);

/* Counting sort of `species` by element, ties by particle id; drops
 * absorbed particles (ParticleBundle%DelOne swap-with-last, ParticleBundle.f90:120-127). */
int pic_sort_particles(int32_t species);

/* MoveAll (MCCInterface.f90:574-640) -> MoveOne (IMPIC/MoveOne.f90) with
 * Get_ParticleEField_PPR (PPR/Get_ParticleEField_PPR.f90) and
 * AdjustParticleBoundary (MCCInterface.f90:217-534).  push_flag as MoveAll.
 * On an axisymmetric mesh (vx, vy, vz) = (v_z, v_r, v_theta) in the
 * particle's own frame (MoveOne.f90:213-263 without the stored angle). */
int pic_move_all(int32_t species, int32_t push_flag);

/* GetParChg_2D (PIC/GetParChg_2D.f90:1-911): locate, int64 fixed-point
 * bilinear deposit (r-weighted for delta 1, GetParChg_2D.f90:803-821),
 * normalisation by the dual volume.  delta must be the mesh's.  rho_out
 * (host, [nodes]) may be NULL. */
int pic_get_par_chg(int32_t delta, double *rho_out);

/* Time-dependent potential on the Dirichlet wall x = xmin (wall 0) or
 * x = xmax (wall 1): at every solve its nodes (corners included, as the mesh
 * builder assigns them; conductor-object nodes excluded) take their static
 * value + amplitude * sin(2 pi frequency_hz * time * t_ref + phase), time
 * being pic_ife_solve's argument or step * dt in pic_step.  amplitude in
 * Phi_ref units; 0 switches it off and restores the static values.  The
 * reference's bc_value(1) = V/Phi_ref*SIN(2*Pi*Frequency*time*time_ref) on
 * the left boundary (IFE_Solve_2D.f90:104-121, commented out there).
 * Deviation: the reference REPLACES the left wall's value by the sine (no
 * static offset) and drives only the left wall; here the sine is ADDED to the
 * wall's static value and either x wall may be driven.  The two agree when
 * the driven wall's static value is 0, as on the r-z electrode deck; give the
 * wall a static value of 0 in the deck to get the reference's form.
 * PIC_ERR_ARG for another wall or one that is not Dirichlet. */
int pic_set_wall_rf(int32_t wall, double amplitude, double frequency_hz, double phase);

/* IFE_Solve_2D (IFE-Rectangular/IFE_Solve_2D.f90:1-260) -> MY_JPCG_Solver ->
 * MY_PCG (IFE-Solver/MY_PCG.f90).  phi_inout (host, [nodes]) may be NULL:
 * then the device phi is the warm start and stays on the device. */
int pic_ife_solve(double *phi_inout, double time, pic_solve_stats *stats);

/* GetEField_SIDG_PPR (PPR/GetEfield_SIDG_PPR.f90:153-304): per-node
 * quadratic recovery, efx = -d(phi)/dx.  Outputs may be NULL. */
int pic_get_efield_ppr(double *efx_out, double *efy_out);

/* MCCEntrance / MCC (MCCInterface.f90:560-569, mc/MCCPublic.F90:35-111). */
int pic_mcc(uint64_t step, pic_mcc_stats *stats);

/* One explicit step in the order of Main_IFE_Test_2.f90:329-341 with MCC after
 * the field solve (MCC_jw/code/OneStep.F90:50-67): fused push+locate+deposit,
 * RHS + PCG, PPR, MCC; counting sort every sort_interval steps. */
int pic_step(uint64_t step, pic_step_stats *stats);

/* Field readback (host, [nodes]).  which: 0 rho, 1 phi, 2 efx, 3 efy,
 * 4+s rho_s of species s, 8+s Ek_s of species s (mean energy per particle,
 * eV), 12..16 coef_ppr(2..6,:), 20 the solver's right-hand side b, 24+s
 * Ek_tot of species s (energy density, normalised like rho_s:
 * GetParChg_2D.f90:895-904).  Ek_s and Ek_tot are those of the last step
 * that deposited energy (pic_params.diag_interval). */
int pic_get_field(int32_t which, double *host_out);
/* Field upload (host, [nodes]): which 1 phi, 2 efx, 3 efy, 12..16 coef_ppr. */
int pic_set_field(int32_t which, const double *host_in);

/* Asynchronous readback of the fields a step leaves (host, [nodes] each;
 * any pointer may be NULL): phi, rho, efx, efy are copied in that order on
 * a copy stream of their own and the call returns at once, so the copies
 * run while the caller's next pic_step pushes the particles.  Every later
 * call that writes one of these fields on the device first waits for its
 * copy (pic_set_field of phi for the phi copy only).  The host arrays must
 * stay valid, and are complete only after pic_wait_fields; they should be
 * page-locked (cudaHostAlloc), or the copies cannot overlap anything.
 * Copy engines serve one direction in order, whatever the stream, so the
 * step reads its counters through a mapped page-locked mirror and clears
 * its accumulators with kernels: these copies, or a caller's own on another
 * stream, run alongside the step instead of holding its start back.
 * Replaces the synchronous per-field reads the reference's caller does
 * after `IFE_Solve_2D` / `GetEField_SIDG_PPR` (Main_IFE_Test_2.f90:329-341)
 * when it does not need the values before its next step. */
int pic_get_fields_async(double *rho_out, double *phi_out, double *efx_out, double *efy_out);
/* Waits for the copies of pic_get_fields_async and pic_set_field_async; the
 * library's stream is ordered after them too (a pic_device_timer stop
 * covers them). */
int pic_wait_fields(void);
/* Asynchronous upload of rho (which 0) or phi (which 1) from host [nodes],
 * on the same copy stream, after the copies already queued there (so phi can
 * go back in from the array pic_get_fields_async is filling): the caller's
 * next pic_step pushes its particles meanwhile and its deposit, solve and
 * field recovery wait for the upload; any call that reads or writes the
 * field first waits for it.  The host array must stay unchanged until
 * pic_wait_fields.  The role of the Rho / Phi arguments of `IFE_Solve_2D`
 * (IFE_Solve_2D.f90:1) when the caller keeps the loop going. */
int pic_set_field_async(int32_t which, const double *host_in);

/* Device pointers of the particle SoA, for zero-copy callers on the same
 * device.  Order: x, y, vx, vy, vz (double*: absolute normalised position and
 * velocity), loc (int32*), id (uint32*).  Only the PIC_PREC_FP64 layout is
 * handed out.  With PIC_PREC_MIXED the same storage holds FP32 data (x, y the
 * offsets inside element loc in element widths, [0, 1]; vx, vy, vz FP32
 * velocities), which a caller expecting doubles would misread, so the call
 * returns PIC_ERR_STATE there; pic_download_particles converts that layout
 * back to FP64 positions. */
int pic_particle_device_ptrs(int32_t species, void **ptrs7, int64_t *n_slots);

/* Number of library kernels launched since init (for launch accounting). */
int64_t pic_kernel_launches(void);

/* Device timer on the library's stream: op 0 records the start event,
 * op 1 records the stop event, waits for it and writes the elapsed ms. */
int pic_device_timer(int32_t op, double *ms_out);

/* ---- learned preconditioner hook (flexible CG) ---- */

/* Preconditioner z = M(r) for flexible CG: r and z are device vectors on the
 * full node grid (0 on Dirichlet nodes).  Called on the host between two
 * kernels of pic_ife_solve; it must leave z complete in the order of the
 * library stream (enqueue on pic_cuda_stream(), or synchronise before
 * returning).  Returns 0, or non-zero to make the solve fall back to
 * Jacobi-PCG.  No reference counterpart: MY_PCG (IFE-Solver/MY_PCG.f90) is
 * Jacobi-preconditioned only. */
typedef int (*pic_precond_fn)(const double *r_dev, double *z_dev, void *user);

/* Registers fn (NULL clears it).  With solver PIC_SOLVER_FCG_UNET and a
 * registered fn, pic_ife_solve runs truncated flexible CG (FCG(m), Notay
 * 2000) to the same relative tolerance as MY_PCG, accepted on the true
 * residual b - A x, and falls back to Jacobi-PCG from the current iterate
 * when FCG stalls or fn fails; pic_solve_stats.fallback reports why. */
int pic_set_preconditioner(pic_precond_fn fn, void *user);
/* Selects the linear solver at run time (PIC_SOLVER_*). */
int pic_set_solver(int32_t solver);
/* Directions FCG keeps for A-orthogonalisation, 1..8 (default 4; 1 = FCG(1)). */
int pic_set_fcg_window(int32_t window);
/* With PIC_PREC_MIXED: 1 runs the one-kernel FCG's iterations in FP32 (FP32
 * vectors and coefficients, FP64 dot products and coarse solve) inside an
 * FP64 iterative refinement x += e, r = b - A x until the tolerance holds on
 * the FP64 residual; 0 (default) keeps the iterations in FP64. */
int pic_set_fcg_inner(int32_t fp32);
/* Preconditioner of flexible CG as a composition of stages:
 *   1. damped-Jacobi pre-smoothing        z1 = omega D^-1 r          (smoothing)
 *   2. Galerkin coarse correction         z2 = z1 + P Ac^-1 P^T (r - A z1)
 *   3. learned correction (the callback)  z3 = z2 + fn(r - A z2)     (learned)
 *   4. damped-Jacobi post-smoothing       z  = z3 + omega D^-1 (r - A z3)
 * Defaults: smoothing off, learned on, no coarse space, so registering fn
 * alone gives M = fn. */
int pic_set_precond_stages(int32_t smoothing, double omega, int32_t learned);
/* Builds the coarse space of stage 2 as a two-level method: bilinear
 * prolongation P from a uniform coarse grid whose spacing is about
 * min(cells)/coarse_cells nodes (a divisor of both cell counts), Ac = P^T A P
 * from mesh's stiffness matrix, inverted on the device and applied from a
 * scaled FP16 copy (at most 9000 coarse nodes).  coarse_cells = 0 removes it.
 * Replaces a multigrid hierarchy. */
int pic_coarse_setup(const pic_mesh_desc *mesh, int32_t coarse_cells);
/* Builds the coarse space of stage 2 as a geometric multigrid V-cycle: the
 * grid halved (every second node) until at most max_coarse_nodes remain
 * (nnx-1 and nny-1 need enough factors of 2; at most 9000 nodes), Galerkin
 * operators A_{l+1} = P^T A_l P of bilinear P from mesh's stiffness matrix,
 * one damped-Jacobi sweep (stage 1's omega) down and up at each level, the
 * coarsest level solved with its dense inverse (FP16 copy, FP64
 * accumulation).  max_coarse_nodes <= 0 removes it.  Replaces a two-level
 * coarse space.  No reference counterpart (MY_PCG is Jacobi-PCG). */
int pic_multigrid_setup(const pic_mesh_desc *mesh, int32_t max_coarse_nodes);
/* z = M(r) (full != 0), or stages 1-2 only (full == 0): the classical part
 * whose residual r - A z is the learned correction's input.  Device vectors,
 * enqueued on the library stream. */
int pic_precond_apply(int32_t full, const double *r_dev, double *z_dev);
/* The library's CUDA stream (a cudaStream_t) for callers that enqueue work
 * in its order. */
int pic_cuda_stream(void **stream);
/* out = A v on the full grid with the solver's operator (Dirichlet rows give
 * 0); device vectors, enqueued on the library stream. */
int pic_apply_operator(const double *v_dev, double *out_dev);
/* Device pointers of the solver's right-hand side b and potential phi
 * (full grid), valid until pic_finalize. */
int pic_solver_vectors(double **b_dev, double **phi_dev);

/* ---- diagnostics (computed on the device) ---- */

/* Average_x (In-Output/Output_To_Tecplot_IJK_2D.f90:166-226, the column
 * profiles of the field output): for each mesh column x = x_i the mean over
 * its nodes, in the file's output scaling.  out is host memory,
 * [(3 + 3*n_species) * nnx], column-major by quantity: x*L_ref, phi*Phi_ref,
 * rho*n_ref, then rho_s*n_ref, Ek_s and Ek_tot of each species in species
 * order (the reference's nine columns for two species).  Each column is summed
 * in node order (j ascending), as the reference does. */
int pic_average_x(double *out);

/* Output_Energy.f90:41-71: counts of one species' live particles whose
 * energy (eV, EnergyParticleOne with VFactor, base/ParticleOne.f90:235-244)
 * lies in (E_max*(b-1)/N, E_max*b/N] and whose vx lies in
 * (V_max*(b-1-N/2)/N, V_max*(b-N/2)/N], b = 1..N (0-based arrays here), with
 * the reference's edge arithmetic.  The reference uses N = 100, E_max = 5 eV
 * and V_max = 10, 0.1, 0.01 by species; dN/dE = 10*count/n_ini is the
 * caller's.  count_e, count_vx: host [nbins].  1 <= nbins <= 4096. */
int pic_energy_spectrum(int32_t species, int32_t nbins, double e_max_ev, double v_max,
                        int64_t *count_e, int64_t *count_vx);

/* OUTPUT_velocity.f90:48-103: one species' live particles binned by x column
 * b = min(max(floor(x), 0), nbins-1) (the reference uses 1024); per column
 * the count, the drift velocity (mean of vx, vy, vz; 0 for an empty column)
 * and the thermal velocity sqrt(mean (v - drift)^2).  count: host [nbins];
 * drift, thermal: host [3][nbins] (vx, vy, vz).  FP64 sums (the reference
 * sums in FP32); their order varies from call to call, so the last bits
 * can.  1 <= nbins <= 2048. */
int pic_velocity_moments(int32_t species, int32_t nbins, int64_t *count, double *drift,
                         double *thermal);

/* ---- allocation-free deposit ---- */

/* Largest mesh (nnx*nny nodes) pic_deposit_noalloc accepts: its int64
 * accumulator is a fixed 4 MiB __device__ array. */
#define PIC_NOALLOC_MAX_NODES 524288

/* Charge density of one species, like the per-species rho_s of
 * pic_get_par_chg, for callers that may not allocate device memory (their
 * device memory comes from an arena owned by someone else, or they run a
 * loop that must not pay cudaMalloc's implicit synchronisation).  No
 * counterpart in the reference: it exists only for such callers.
 *
 * Needs no pic_init.  x, y (and loc, may be NULL; loc < 0 skips a particle),
 * cell_volume ([nnx*nny]) and rho_out ([nnx*nny]) are DEVICE pointers of the
 * current device; stream is a cudaStream_t (NULL: default stream).  The call
 * only enqueues work: synchronise the stream before reading rho_out.
 * Allocates and frees nothing.  The scratch is one file-scope __device__
 * array shared by every call on a device: calls that overlap on the GPU
 * (different streams, or several host threads) race on it.  The first call
 * on a device looks up the array's device address (cudaGetSymbolAddress); make
 * that first call before any stream capture.  The address is kept for the
 * life of the process: after a cudaDeviceReset of that device, unload and
 * reload the library before calling again.  Meshes above
 * PIC_NOALLOC_MAX_NODES nodes are rejected with PIC_ERR_ARG.
 *
 * Scope: Cartesian meshes (delta 0) and FP64 absolute positions.  It matches
 * pic_get_par_chg's rho_s bit for bit only on that path: it has no r-weighted
 * (delta 1) weights, axis-row factor or L_ref^3 normalisation, and it reads
 * x, y as doubles, so the FP32 offsets of a PIC_PREC_MIXED context are not
 * valid input (pic_particle_device_ptrs refuses them). */
int pic_deposit_noalloc(int32_t nnx, int32_t nny, double xmin, double xmax, double ymin,
                        double ymax, int64_t n, const double *x, const double *y,
                        const int32_t *loc, const double *cell_volume, double weight_charge,
                        double L_ref, double n_ref, double *rho_out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* PICGPU_H */
