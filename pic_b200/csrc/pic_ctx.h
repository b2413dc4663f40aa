// pic_ctx.h -- device context of libpicgpu (internal).
#ifndef PIC_CTX_H
#define PIC_CTX_H

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

#include "../../include/picgpu.h"
#include "mg_dev.h"
#include "pic_common.h"
#include "pic_mcc_kin.h"

namespace pic {

void set_error(const std::string &msg);
int cuda_fail(cudaError_t e, const char *where);
extern long long g_launches;

#define PIC_CUDA(call)                                      \
  do {                                                      \
    cudaError_t _e = (call);                                \
    if (_e != cudaSuccess) return ::pic::cuda_fail(_e, #call); \
  } while (0)

#define PIC_LAUNCHED()                                          \
  do {                                                          \
    ++::pic::g_launches;                                        \
    cudaError_t _e = cudaPeekAtLastError();                     \
    if (_e != cudaSuccess) return ::pic::cuda_fail(_e, "launch"); \
  } while (0)

// Mesh geometry passed by value to kernels.
struct MeshK {
  int nnx, nny, nex, ney;
  double xmin, xmax, ymin, ymax, hx, hy;
  uint32_t ney_magic;             // floor(2^32 / ney) + 1, for the element -> column split
  const double *xs, *ys;          // node coordinates (x_s + h_x*(i))
  const int32_t *element_index;   // [ne]
  const int32_t *node_index;      // [nn]
  const uint8_t *elem_near;       // [ne] 1: the element's box meets an object's box
};

struct ObjK {
  int n;
  pic_object o[PIC_MAX_OBJECTS];
  // per object, computed on the host: cos/sin of the ellipse angle (the
  // host's libm, as the oracle) and the half-width of a box that holds it
  double ca[PIC_MAX_OBJECTS], sa[PIC_MAX_OBJECTS], half[PIC_MAX_OBJECTS];
};

struct Species {
  // With PIC_PREC_MIXED (f32) the five value arrays x, y, vx, vy, vz hold FP32
  // data in the first half of their storage: x, y are the offsets inside the
  // element loc (in element widths, [0, 1]), vx, vy, vz the velocities.  The
  // FP64 layout is used only to stage uploads and downloads.
  bool f32 = false;
  double charge = 0, mass = 0, weight = 0, qm = 0;
  int64_t capacity = 0, n_slots = 0, n_live = 0;
  uint32_t next_id = 0;
  double *x = nullptr, *y = nullptr, *vx = nullptr, *vy = nullptr, *vz = nullptr;
  int32_t *loc = nullptr;
  uint32_t *id = nullptr;
  // second buffer for the counting sort
  double *x2 = nullptr, *y2 = nullptr, *vx2 = nullptr, *vy2 = nullptr, *vz2 = nullptr;
  int32_t *loc2 = nullptr;
  uint32_t *id2 = nullptr;
  // deposit accumulators (fixed point) and normalised per-species fields:
  // rho_s charge density, ek_s mean energy per particle (eV), ek_tot energy
  // density (GetParChg_2D.f90:880-904; ek_s and ek_tot on energy steps)
  unsigned long long *q_acc = nullptr, *e_acc = nullptr;
  double *rho_s = nullptr, *ek_s = nullptr, *ek_tot = nullptr;
  // MCC
  bool has_mcc = false;
  pic_mcc_table tab;
  double *prob = nullptr;  // [n_sigma*n_reaction]
};

struct PcgState {
  double rho, rho0, alpha, beta, normR, normRHS, tol2;
  int iter, maxit, done, ierr;
  unsigned int ticket;
  int pad;
};

// Flexible-CG scalars, resident on the device during a solve.
#define PIC_FCG_MAX_WINDOW 8
struct FcgState {
  double pq, pr, alpha, rr, rhs, tol2, best;
  double beta[PIC_FCG_MAX_WINDOW];     // against the last `count` directions, newest first
  double pq_hist[PIC_FCG_MAX_WINDOW];  // P_j.Q_j per ring slot
  int iter, maxit, done, ierr, best_iter, count, stall_window;
  unsigned int ticket;
};

struct Ctx {
  bool inited = false;
  MeshK m;
  int64_t nn = 0, ne = 0;
  pic_params P;
  double L_ref = 0, t_ref = 0, v_ref = 0, phi_ref = 0;
  cudaStream_t st = nullptr;
  cudaStream_t st2 = nullptr;  // the step's field recovery, alongside its MCC
  // asynchronous field readback (pic_get_fields_async): the copy stream, the
  // event it starts after, one event per field (0 rho, 1 phi, 2 efx, 3 efy)
  // and the fields whose copies may still run
  cudaStream_t st_copy = nullptr;
  cudaEvent_t ev_copy_start = nullptr, ev_field[4] = {nullptr, nullptr, nullptr, nullptr};
  unsigned copy_pending = 0;
  cudaEvent_t step_ev[10] = {};                 // pic_step's phase events, created once
  unsigned long long *h_counters = nullptr;     // mapped pinned mirror of d_counters
  unsigned long long *hd_counters = nullptr;    // its device address (a kernel writes it)
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // mesh
  double *d_xs = nullptr, *d_ys = nullptr;
  int32_t *d_element_index = nullptr, *d_node_index = nullptr, *d_node_type = nullptr;
  uint8_t *d_elem_near = nullptr;
  double *d_phi_dir = nullptr, *d_cell_volume = nullptr, *d_rhs_fix = nullptr;
  double *d_mass_q1 = nullptr, *d_ife_mass = nullptr;
  double *d_mass_rows = nullptr;  // delta = 1 only
  bool axi = false;               // delta = 1: r-z push and deposit
  int32_t *d_xt_ptr = nullptr, *d_xt_col = nullptr;  // per unknown row, 0-based node columns
  double *d_xt_val = nullptr;
  // PCG operator: row kind per node (-1 Dirichlet, 0..n_mat-1 stencil, >= n_mat explicit row)
  int32_t *d_row_kind = nullptr;
  int32_t *d_ex_cnt = nullptr, *d_ex_col = nullptr;  // explicit rows: count + 9 padded slots
  double *d_ex_val = nullptr;
  float *d_ex_val32 = nullptr;     // FP32 copy (inner iterations of the mixed-precision FCG)
  float *d_fcg32 = nullptr;        // mixed-precision FCG: 11 FP32 vectors, allocated on first use
  int fcg_inner32 = 0;             // mixed precision: FP32 inner FCG in FP64 refinement (pic_set_fcg_inner)
  int n_mat = 0;
  double h_stencil[16][9];
  double *d_diag = nullptr;  // [nn], 1 on Dirichlet nodes
  // PPR
  int32_t *d_ppr_kind = nullptr;  // 0 regular 3x3, 1 explicit, 2 none
  int32_t *d_ppr_ptr = nullptr, *d_ppr_nodes = nullptr;  // explicit patches
  double *d_ppr_rows = nullptr;  // [5][n] per explicit node, at 5*ptr
  double *d_ppr_h = nullptr;     // h per node
  double h_ppr_reg[5][9];
  // fields
  double *d_phi = nullptr, *d_rho = nullptr, *d_efx = nullptr, *d_efy = nullptr;
  double2 *d_efxy = nullptr;  // {efx, efy} per node, written with them (the FP64 push's gather)
  double *d_coef = nullptr;  // [5][nn] coef_ppr(2..6,:)
  bool mixed = false;        // PIC_PREC_MIXED
  float *d_coef32 = nullptr; // mixed: per node {c2, c3, c4, c5, c6, 0, 0, 0} in FP32 (32 B records)
  // PCG vectors (full grid)
  double *d_b = nullptr, *d_x = nullptr, *d_r = nullptr, *d_w = nullptr, *d_p[2] = {nullptr, nullptr},
         *d_q = nullptr;
  double *d_part = nullptr;  // block partials [3][nblk]
  PcgState *d_pcg = nullptr;
  int red_blocks = 0;
  int coop_grid = 0;               // CTAs of the persistent PCG (0: two-kernel loop)
  int fcg_coop_grid = 0;           // CTAs of the persistent FCG (0: graph-launched iterations)
  int smem_grid = 0;               // CTAs of the shared-memory-resident PCG (0: not eligible)
  bool ex_local = true;            // every explicit row stays inside its 3x3 neighbourhood
  size_t smem_bytes = 0;
  unsigned int *d_bar = nullptr;   // grid barrier: count, generation, error flag
  // flexible CG with a registered preconditioner
  pic_precond_fn precond = nullptr;
  void *precond_user = nullptr;
  int solver = PIC_SOLVER_JPCG;
  double *d_z = nullptr, *d_dot = nullptr;  // preconditioned residual, dot results [2]
  unsigned int *d_dot_ticket = nullptr;
  FcgState *d_fcg = nullptr;
  int fcg_window = 4;                       // FCG(m) directions kept
  double *d_fcg_P = nullptr, *d_fcg_Q = nullptr, *d_fcg_part = nullptr;  // allocated on first use
  int fcg_last_iters = 8;                   // iterations of the previous FCG solve (chunk sizing)
  int64_t fcg_precond_calls = 0;
  // composite preconditioner of FCG (precond.cu)
  int pc_sweeps = 0;                        // damped-Jacobi pre/post smoothing on (1) or off (0)
  double pc_omega = 2.0 / 3.0;
  int pc_learned = 1;                       // apply the registered callback as stage 3
  int pc_cs = 0, pc_ncx = 0, pc_ncy = 0;    // coarse spacing in nodes (0: no coarse space)
  double *d_pc_t = nullptr, *d_pc_y = nullptr, *d_pc_za = nullptr, *d_pc_dinv = nullptr;
  __half *d_pc_ainv = nullptr;             // coarse inverse / pc_ainv_scale, FP16, row-major, rows of pc_ainv_ld
  double pc_ainv_scale = 1.0;
  int pc_ainv_ld = 0;                       // coarse inverse row length: coarse nodes rounded up to 8
  double *d_pc_rc = nullptr, *d_pc_ec = nullptr;
  MgK mg{};                                 // multigrid hierarchy (mg.L = 0: none)
  int push_stages = 4, push_grid = 0;       // tiled mixed push stages (0: one particle per thread)
  int push_minb = 5;                        // resident CTAs per SM the 4-stage push is built for
  int push64_grid = 0;                      // tiled FP64 push: persistent CTAs (0: direct kernel)
  int push64_default = 2;                   // bulk-tiled FP64 push unless PIC_PUSH64_TILED=0 or 1
  bool push64_bulk = false;                 // tiles bulk-copied (PIC_PUSH64_TILED=2)
  int push64_minb = 4;                      // resident CTAs per SM the Cartesian bulk push is built for
  bool push_bulk = false;                   // mixed-precision tiles bulk-copied (PIC_PUSH_BULK=1)
  int push_bulk_default = 1;
  long long push_wait_limit = 1ll << 22;    // polls of a tile's mbarrier before the push gives up
  int push_skip_copies = 0;                 // test hook: the bulk pushes issue no tile copies
  // CUDA graphs of one FCG iteration: [0] stage A, [1 + slot] stage B + FCG
  // kernels of ring slot `slot`; rebuilt when the configuration key changes
  cudaGraphExec_t fcg_graph[2 + PIC_FCG_MAX_WINDOW] = {};
  long long fcg_graph_launches[2 + PIC_FCG_MAX_WINDOW] = {};
  unsigned long long fcg_graph_key = 0, fcg_graph_gen = 1;
  int fcg_graphs = 1;                       // capture iterations (PIC_FCG_GRAPHS=0 turns it off)
  long long pcg_spin_limit = 1ll << 24;
  unsigned int pcg_bar_extra = 0;
  int ebc_dirty = 1;
  // species
  int ns = 0;
  Species sp[PIC_MAX_SPECIES];
  // scratch
  int32_t *d_cell_count = nullptr, *d_cell_start = nullptr, *d_cell_fill = nullptr;
  int32_t *d_perm = nullptr, *d_perm2 = nullptr;
  uint32_t *d_sort_id = nullptr;
  int32_t *d_scan_blk = nullptr;
  unsigned long long *d_counters = nullptr;  // misc device counters
  // MCC
  pic_gas gas;
  bool mcc_ready = false;
  uint32_t *d_hist = nullptr;          // [65536] per species (the full selection uses species 0's)
  int32_t *d_sel = nullptr;            // selected slots
  uint64_t *d_cand = nullptr;          // candidates (key<<32 | id), slot in d_cand_slot
  int32_t *d_cand_slot = nullptr;
  int64_t mcc_cap = 0;                 // d_sel entries; ionisation entries per species
  int64_t cand_cap = 0;                // d_cand, d_cand_slot entries
  int64_t *d_mcc_misc = nullptr;       // [16] counters per species
  uint64_t *d_mlist_key = nullptr;     // bounded selection: (key << 32 | id) below the bound
  int32_t *d_mlist_slot = nullptr;     //   and their slots; mlist_cap entries per species
  int64_t mlist_cap = 0;
  // the bounded selection of this step's MCC, built by the push
  // (sel_step = the step it is for; sel_push: run_push passes the sinks)
  bool mcc_push_select = true;  // PIC_MCC_PUSH_SELECT=0: off
  MccSink sel_sink[PIC_MAX_SPECIES];
  uint64_t sel_step = ~0ull;
  bool sel_push = false;
  int mcc_full = 0;                    // 1: always the full-histogram selection
  double mcc_bound_scale = 1.0;        // test hook: < 1 forces the bounded selection's fallback
  int64_t *d_msel = nullptr;           // [8] per species: list count, keys below the bound, b*,
                                       //   count below b*, selection held
  int64_t *d_ion_parent = nullptr;     // ionising parents: (id<<32 | slot), mcc_cap per species
  double *d_ion_data = nullptr;        // per ionisation: new e- v(3), ion v(3)
  void *h_fcg = nullptr;               // pinned FcgState of the fused persistent FCG
  size_t fcg_smem_set = 0;             // dynamic shared memory the FCG kernel was opened to
  int fcg_fused = 1;                   // PIC_FCG_FUSED=0: set-up and judge by separate kernels
  int32_t *d_mcc_pslot = nullptr;      // created particles: parent slots, velocities (e, ion), rank order
  int32_t *d_ion_order = nullptr;
  double *d_mcc_vel = nullptr;
  int64_t mcc_new_cap = 0;
  int64_t step_count = 0;
  // time-dependent wall potential (pic_set_wall_rf): the Dirichlet nodes of
  // the lines x = xmin (0) and x = xmax (1) other than conductor nodes, their
  // static values, and whether every node of the line is Dirichlet
  std::vector<int32_t> rf_line[2];
  std::vector<double> rf_base[2];
  bool rf_ok[2] = {false, false};
  int rf_wall = -1;  // -1: off
  int rf_count = 0;
  double rf_amp = 0.0, rf_omega = 0.0, rf_phase = 0.0;  // omega: radians per normalised time
  int32_t *d_rf_nodes = nullptr;
  double *d_rf_base = nullptr;
};

extern Ctx g;

// kernels launched from other translation units
int launch_locate(Species &s, int64_t begin, int64_t end);
int sort_species(int sidx);
int mcc_run(uint64_t step, pic_mcc_stats *stats, bool prepared = false);
int mcc_prepare(uint64_t step);
int fields_fence(unsigned mask);  // the library stream waits for queued copies of fields in mask
int zero_async(void *p, size_t bytes, cudaStream_t st);  // zero fill by a kernel (bytes, p: multiples of 4)
int launch_spmv(const double *v, double *out);  // out = A v (solver operator)
int coarse_setup(const pic_mesh_desc *mesh, int coarse_cells);
int precond_apply(int full, const double *r, double *z);
int coarse_correct(const double *t, double *z, int assign);
int mg_setup(const pic_mesh_desc *mesh, int max_coarse_nodes);
int mg_correct(const double *t, double *z, int assign);
inline bool coarse_on() { return g.pc_cs > 0 || g.mg.L > 1; }
int precond_learned_on();
int precond_prepare();
int precond_callback();
void precond_free();
void diag_free();

inline int blocks_for(int64_t n, int threads) { return (int)((n + threads - 1) / threads); }

}  // namespace pic

#endif
