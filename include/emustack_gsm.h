/*
 * emustack_gsm.h -- C ABI of the B200-native EMUstack GSM stage.
 *
 * The generalised scattering-matrix (GSM) stage of EMUstack computes, for a
 * stack of homogeneous films and periodic nanostructured layers, the
 * interface scattering matrices, the net reflection/transmission matrices
 * R_net / T_net and the energy fluxes (per-layer absorptance a_list,
 * t_list, r_list).  In the reference this is Python + numpy/LAPACK
 * (backend/stack.py, backend/mode_calcs.py) fed by the Fortran overlap
 * integrals backend/fortran/J_overlap.f and J_dagger_overlap.f (bound to
 * Python through f2py).  Every entry point below replaces one of those
 * pieces; the citation beside each names the reference interface it stands
 * in for (paths relative to the EMUstack source tree).
 *
 * Conventions
 *   - Every function returns an int status (EMU_OK = 0); none aborts.
 *   - Pointers named d_* are CUDA device pointers; h_* are host pointers.
 *   - Complex numbers are interleaved (re, im) doubles (emu_c128), the layout
 *     of numpy complex128 and std::complex<double>.  Matrices are row-major
 *     (C order), batch index outermost.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default
 *     stream).  Calls are asynchronous on that stream unless stated.
 *   - The caller owns every buffer.  Functions that need scratch memory take
 *     (d_workspace, workspace_bytes) and have a *_workspace_size query.
 */
#ifndef EMUSTACK_GSM_H
#define EMUSTACK_GSM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define EMU_OK 0
#define EMU_E_ARG 1          /* null pointer, bad enum, inconsistent sizes  */
#define EMU_E_SHAPE 2        /* unsupported or inconsistent dimensions      */
#define EMU_E_SINGULAR 3     /* exactly singular matrix in a solve          */
#define EMU_E_NONFINITE 4    /* NaN / Inf produced                          */
#define EMU_E_WORKSPACE 5    /* workspace too small                         */
#define EMU_E_TIMEOUT 6      /* a bounded device-side wait gave up          */
#define EMU_E_CUDA 7         /* CUDA launch / runtime error                 */
#define EMU_E_UNSUPPORTED 8

/* Polarisations of the specular incidence vector
 * (backend/mode_calcs.py:220-250 Anallo.specular_incidence). */
#define EMU_POL_TE 0
#define EMU_POL_TM 1
#define EMU_POL_UN 2
#define EMU_POL_RCIRC 3
#define EMU_POL_LCIRC 4
#define EMU_POL_INCOMING (-1) /* use the caller's incoming amplitudes        */

/* Per-point status bits written by emu_film_stack_batch. */
#define EMU_PT_WOOD_AIR 1u        /* air reference hit a Wood anomaly        */
#define EMU_PT_WOOD_LAYER 2u      /* some layer hit a Wood anomaly           */
#define EMU_PT_NO_PROP_SUB 4u     /* no propagating orders in the substrate  */
#define EMU_PT_NO_PROP_SUP 8u     /* no propagating orders in the superstrate*/
#define EMU_PT_NONFINITE 16u      /* NaN / Inf in an output of this point    */

typedef struct {
  double re, im;
} emu_c128;

/* Library version (major*10000 + minor*100 + patch). */
int emu_version(void);

/* Process-wide choice of the dense interface and cascade paths (no
 * counterpart in the reference): 0 automatic (by matrix size and batch),
 * 1 one CTA per problem, 2 every step spread over many CTAs.  Results are
 * bit-identical; only speed differs.  Returns the previous value, or -1 for
 * an invalid mode.  An EmuStackDense.mode other than 0 takes precedence. */
int emu_set_dense_mode(int mode);

/* Human-readable name of a status code. */
const char *emu_status_string(int status);

/* Number of CUDA kernels this library launched since load (all entry points,
 * all devices).  Host-side counter, incremented at each launch. */
long long emu_launch_count(void);

/* ------------------------------------------------------------ a1: orders
 * Plane-wave diffraction orders inside the disc
 *   (px/d)^2 + (py/dy)^2 <= (max_order / max(d, dy))^2,
 * px outer, py inner, evaluated in IEEE double without contraction so that
 * the set matches the reference exactly (including orders dropped by
 * rounding on the circle).
 * Replaces Modes.calc_2d_grating_orders / calc_1d_grating_orders
 * (backend/mode_calcs.py:55-74) and the order loop of pw_ordering
 * (backend/fortran/pw_ordering.f:54-78).
 * h_px / h_py may be NULL to query the count; capacity is their length.
 * world_1d != 0 gives px = -max_order..max_order and py = 0. */
int emu_grating_orders(int max_order, double period, double period_y, int world_1d,
                       int32_t *h_px, int32_t *h_py, int capacity, int *h_count);

/* ------------------------------------------- a2: analytic film modes
 * k_z of one homogeneous film per point, sorted: the air reference sorts by
 * -Re k_z + Im k_z (d_sort_in == NULL, backend/mode_calcs.py:164-171), any
 * other film applies the air's sort order (d_sort_in = the air's d_sort_out,
 * backend/mode_calcs.py:172-175).  Includes the Wood-anomaly retry with
 * k_parallel * (1 - 1e-9) (backend/mode_calcs.py:147-162), the specular
 * order and the number of propagating orders (k_z.imag == 0).
 * Replaces Anallo.calc_kz (backend/mode_calcs.py:116-186).  Ties in the air
 * sort keys (only when a k_parallel component is exactly zero) are ranked by
 * order index, as numpy's argsort ranks them for up to 16 orders; tied
 * orders have identical k_z. */
typedef struct {
  int n_points;            /* B films (each with its own wavelength)        */
  int n_pw;                /* Npw                                           */
  int world_1d;
  double period, period_y; /* nm                                            */
  const int32_t *d_px;     /* [Npw]                                         */
  const int32_t *d_py;     /* [Npw]                                         */
  const double *d_wl_nm;   /* [B]                                           */
  const double *d_k_pll;   /* [B][2] nm^-1                                  */
  const emu_c128 *d_n;     /* [B] refractive index (loss applied)           */
  const int32_t *d_sort_in;/* [B][Npw] or NULL (air reference)              */
  emu_c128 *d_kz;          /* [B][Npw] sorted k_z (required)                */
  double *d_alphas;        /* [B][Npw] unsorted alphas (optional)           */
  double *d_betas;         /* [B][Npw] unsorted betas (optional)            */
  int32_t *d_sort_out;     /* [B][Npw] sort order used (optional)           */
  int32_t *d_specular;     /* [B] (optional)                                */
  int32_t *d_num_prop;     /* [B] (optional)                                */
  int32_t *d_wood;         /* [B] 1 if the Wood retry was taken (optional)  */
} EmuAnalloModes;

int emu_anallo_modes(const EmuAnalloModes *p, void *stream);

/* ------------------------------------- a2-a4, a7, a9, a10: film stacks
 * Batched solve of all-film stacks: every layer is a homogeneous film, so
 * every interface, propagation and cascade matrix is diagonal and the stage
 * reduces to independent scalar recursions per plane-wave order.  One
 * launch computes, for each spectral point b:
 *   - the air reference's k_z, its sort order (argsort(-Re kz + Im kz)),
 *     the specular order and the propagating counts
 *     (backend/mode_calcs.py:116-186, backend/objects.py:1745-1777);
 *   - every film's k_z = sqrt(k^2 - alpha^2 - beta^2) with the Wood-anomaly
 *     retry and impedances Z (backend/mode_calcs.py:116-218);
 *   - the air/film Fresnel interfaces (backend/mode_calcs.py:451-477);
 *   - the cascade R_net, T_net with optional shears
 *     (backend/stack.py:196-287, backend/mode_calcs.py:76-87);
 *   - the energy fluxes and a_list / t_list / r_list (backend/stack.py:289-426).
 * Layers are ordered bottom (substrate, index 0) to top (superstrate,
 * index L-1) as in Stack(layers).  n is the refractive index with the
 * layer's `loss` flag already applied (imaginary part zeroed when False).
 */
typedef struct {
  int n_points;          /* B                                               */
  int n_layers;          /* L >= 2, substrate and superstrate included      */
  int n_pw;              /* Npw, orders per polarisation (P = 2 Npw)        */
  int world_1d;          /* 1: 1D order set, beta = beta0                   */
  double period;         /* nm                                              */
  double period_y;       /* nm                                              */
  const int32_t *d_px;   /* [Npw] orders from emu_grating_orders            */
  const int32_t *d_py;   /* [Npw]                                           */
  const double *d_wl_nm; /* [B] wavelengths (nm)                            */
  const double *d_k_pll; /* [B][2] k_parallel (nm^-1), Light.k_pll          */
  const emu_c128 *d_n;   /* [B][L] refractive indices                       */
  const double *d_heights_nm; /* [L-2] or [B][L-2] finite-layer heights     */
  int heights_per_point; /* 0: one height list for all points               */
  int pol;               /* EMU_POL_*                                       */
  const emu_c128 *d_incoming; /* [B][P] when pol == EMU_POL_INCOMING        */
  const double *d_shears;/* [L][2] layer shifts (unit-cell units) or NULL   */
  int shear_ncoord;      /* 1 (1D) or 2                                     */
  /* outputs (required) */
  emu_c128 *d_R_net;     /* [B][P] diagonal of R_net (sorted order)         */
  emu_c128 *d_T_net;     /* [B][P] diagonal of T_net                        */
  double *d_a_list;      /* [B][L-1] per-layer absorptance, total last      */
  double *d_t_list;      /* [B][L-1]                                        */
  double *d_r_list;      /* [B]                                             */
  uint32_t *d_flags;     /* [B] EMU_PT_* bits                               */
  /* optional outputs (NULL to skip) */
  emu_c128 *d_kz;        /* [B][L][Npw] sorted k_z of every layer           */
  emu_c128 *d_layer_rt;  /* [B][L][2][P] R12, T12 diagonals (R21=-R12, T21=T12) */
  emu_c128 *d_vec_coef_down; /* [B][L][P]                                   */
  emu_c128 *d_vec_coef_up;   /* [B][L-1][P]                                 */
  double *d_fluxes;      /* [B][L+1][2]: down fluxes 0..L-1 (complex), up0  */
  int32_t *d_sort_order; /* [B][Npw] air sort order (argsort result)        */
  int32_t *d_specular;   /* [B] specular order index                        */
  int32_t *d_num_prop;   /* [B][L+1] propagating orders per layer, air last */
  /* launch variant (threads per CTA x minimum CTAs per SM): 0 = 256 x 2
   * (default), 1 = 128 x 4, 2 = 512 x 1, 3 = 256 x 1 (up to 255 registers),
   * 4 = 256 x 3, 5 = 256 x 4 (85 / 64 registers: more resident warps, some
   * values spilled to L1);
   * results are identical, only speed differs (chosen by an autotuner) */
  int variant;
} EmuFilmStackBatch;

/* Workspace: only pol == EMU_POL_INCOMING needs one (B x Npw x L x 160
 * bytes: any order may carry light, and each such order keeps its flux-pass
 * scalars there); for the other polarisations the size is 0 and d_workspace
 * may be NULL. */
size_t emu_film_stack_workspace_size(const EmuFilmStackBatch *p);
int emu_film_stack_batch(const EmuFilmStackBatch *p, void *d_workspace,
                         size_t workspace_bytes, void *stream);

/* ---------------------------------------- materials: n(lambda) per layer
 * Refractive index of every layer of a stack at a batch of wavelengths,
 * into the [B][L] array the film kernels take: constant, tabulated (linear
 * interpolation with the arithmetic of scipy.interpolate.interp1d, the
 * reference's choice, as scipy 1.18 evaluates it: real indices through
 * numpy.interp (EMU_MAT_TABLE_REAL), complex ones by the weighted form
 * ((x - x0) y1 + (x1 - x) y0) / (x1 - x0) termwise (EMU_MAT_TABLE)) or Drude
 * materials, each with its loss flag applied (imaginary part dropped when
 * loss == 0).  Replaces Material.n
 * (backend/materials.py:31-186) and Anallo.n (backend/mode_calcs.py:186-192)
 * for a sweep.  Wavelengths outside a table set *d_error = 1 and give NaN
 * (the reference raises ValueError there).  At most 32 layers per call. */
#define EMU_MAT_CONSTANT 0
#define EMU_MAT_TABLE 1
#define EMU_MAT_DRUDE 2
#define EMU_MAT_TABLE_REAL 3
typedef struct {
  int kind;              /* EMU_MAT_*                                        */
  int n_rows;            /* table rows (>= 2)                                */
  const double *d_wl;    /* [n_rows] ascending wavelengths (nm), device      */
  const emu_c128 *d_n;   /* [n_rows] refractive indices, device (real part
                            only for EMU_MAT_TABLE_REAL)                      */
  emu_c128 n_const;      /* EMU_MAT_CONSTANT                                 */
  double drude[3];       /* omega_plasma, omega_gamma, eps_inf (EMU_MAT_DRUDE) */
  int loss;              /* 0: imaginary part dropped                        */
} EmuMaterial;

int emu_material_n_batch(const EmuMaterial *h_materials, int n_layers, int n_points,
                         const double *d_wl_nm, emu_c128 *d_n, int32_t *d_error, void *stream);

/* ------------------------------------------ fields from the amplitudes
 * emu_pw_fields: E = (E_x, E_y, E_z) inside one homogeneous layer of B
 * solved stacks, from the layer's plane-wave amplitudes, at the points
 * (x, y, z) in units of the period -- the ThinFilm branch of fields_in_plane
 * (backend/plotting.py:1759-1833) and field_values (plotting.py:2857-2996).
 * z is the distance from the bottom of the layer (from the top of the
 * substrate, into it, for layer 0); a finite layer's height enters the
 * down-going term as exp(-i gamma (z - h)), a semi-infinite layer's as
 * h = 0.  E[b] holds E_x, E_y, E_z, each over the Q points (grid: Q =
 * nx ny nz in [x][y][z] order, the reference's E_x_array[x, y, z]).
 * On a grid the exponentials factor into per-axis tables (x, y and z
 * factors of every order, in the workspace: B (nx + ny + 3 nz) Npw complex
 * values; EMU_E_WORKSPACE when it is missing or short) and the sum over
 * orders is a contraction; points are evaluated term by term.
 * At most 1536 orders per polarisation. */
typedef struct {
  int n_stacks;            /* B                                               */
  int n_pw;                /* Npw orders per polarisation                     */
  int substrate;           /* 1: layer 0 (z -> -z, no upward amplitudes)      */
  int grid;                /* 1: grid x[nx] x y[ny] x z[nz]; 0: nx points     */
  int nx, ny, nz;
  const double *d_alphas;  /* [B][Npw] unsorted (Anallo.alphas)               */
  const double *d_betas;   /* [B][Npw] unsorted (world_1d: beta0 everywhere)  */
  const int32_t *d_sort;   /* [B][Npw] the air reference's sort order         */
  const emu_c128 *d_kz;    /* [B][Npw] sorted k_z (Anallo.calc_kz())          */
  const emu_c128 *d_n;     /* [B] layer index, loss flag applied              */
  const double *d_height;  /* [B] height / period, 0 if semi-infinite; or NULL */
  const emu_c128 *d_vec_coef_down; /* row b at b * vcd_stride: TE then TM     */
  const emu_c128 *d_vec_coef_up;   /* same, or NULL (zero)                    */
  long long vcd_stride, vcu_stride;
  const double *d_x, *d_y, *d_z;   /* units of the period                     */
  emu_c128 *d_E;           /* [B][3][Q]                                       */
  double *d_E_abs;         /* [B][Q] |E|, or NULL                             */
  void *d_workspace;       /* grid: emu_pw_fields_workspace_size bytes        */
  size_t workspace_bytes;
} EmuPwFields;
size_t emu_pw_fields_workspace_size(const EmuPwFields *p);
int emu_pw_fields(const EmuPwFields *p, void *stream);

/* emu_bloch_fields_plane: E at the six P2 nodes of every element of a 2D
 * nanostructured layer at the plane hz (distance from the top of the layer,
 * in units of the period, 0 <= hz <= h; EMU_E_ARG otherwise), from the
 * layer's Bloch-mode amplitudes -- field_value_plane
 * (backend/fortran/field_value_plane.f:6-132), used by fields_in_plane and
 * fields_interpolator_in_plane (backend/plotting.py:1700-1737, 1943-1990).
 * d_E[b][el][node][component] is the routine's m_E(el, node, component). */
typedef struct {
  int n_stacks;            /* B                                               */
  int n_modes;             /* M Bloch modes                                   */
  int n_elements;          /* nel                                             */
  const emu_c128 *d_sol;   /* [B][nel][M][13][3], Fortran sol(3, 13, M, nel)  */
  long long sol_stride;    /* complex values between stacks                   */
  const emu_c128 *d_k_z;   /* [B][M] propagation constants                    */
  const emu_c128 *d_vec_coef; /* [B][2M] vec_coef_down then vec_coef_up       */
  double h, hz;            /* layer height / period; plane                    */
  emu_c128 *d_E;           /* [B][nel][6][3]                                  */
} EmuBlochFieldsPlane;
int emu_bloch_fields_plane(const EmuBlochFieldsPlane *p, void *stream);

/* ------------------------------ serving: device-resident request loop
 * A persistent kernel that solves all-film spectral points as the host
 * writes them into a ring of slots in pinned, device-mapped host memory:
 * no kernel launch per request or batch.  Each request is one
 * Stack(layers).calc_scat(pol) of an all-film stack (backend/stack.py:
 * 162-426; in the reference, one Python call per point) of any shape up to
 * EMU_RING_MAX_LAYERS layers and EMU_RING_MAX_PW orders per polarisation,
 * with a standard polarisation; results are those of emu_film_var_batch
 * for the same point (one warp per request, the same recursion).
 *   create  : allocates the ring (capacity slots of emu_film_ring_slot_bytes()
 *             pinned host bytes) and the device state; the loop ends by itself
 *             idle_seconds after the last request (every device wait is
 *             bounded) and restarts on the next submit.
 *   submit  : copies a request into its slot and wakes the loop; returns a
 *             ticket, or EMU_E_WORKSPACE while the ring is full (poll the
 *             oldest results first).  Thread-safe.  submit_many: the same
 *             for n requests in order, as many as there are free slots
 *             (*n_submitted; EMU_E_WORKSPACE when none).
 *   poll    : 1 and the outputs copied out when the ticket is done, 0 while
 *             pending, a negative status for an unknown or already read
 *             ticket (each result can be read once); poll_many: the same for
 *             n tickets (done[i]), returns how many were read; wait: poll
 *             until done or timeout (-EMU_E_TIMEOUT); ready: 1 when done, 0
 *             while pending, without reading (or consuming) the result.
 *   stop    : ends the loop and waits for it; returns EMU_E_TIMEOUT if a
 *             device wait gave up, else EMU_OK.
 * While the loop runs it holds every SM; other kernels on the device wait
 * for it to end (stop, or idle_seconds without requests). */
#define EMU_RING_MAX_PW 512
#define EMU_RING_MAX_LAYERS 16
typedef struct EmuFilmRing EmuFilmRing;
typedef struct {
  int n_layers, n_pw, world_1d, pol;  /* pol: EMU_POL_TE .. EMU_POL_LCIRC    */
  double period, period_y;            /* nm                                  */
  double wl_nm;
  double k_pll[2];                    /* nm^-1                               */
  const int32_t *h_px, *h_py;         /* [n_pw] orders (emu_grating_orders)  */
  const emu_c128 *h_n;                /* [n_layers] indices, loss applied    */
  const double *h_heights_nm;         /* [n_layers - 2]                      */
} EmuFilmRingRequest;
typedef struct {
  emu_c128 *h_R_net, *h_T_net;        /* [2 n_pw] each, or NULL              */
  double *h_a_list, *h_t_list;        /* [n_layers - 1] each, or NULL        */
  double *h_r_list;                   /* [1] or NULL                         */
  uint32_t *h_flags;                  /* [1] EMU_PT_* or NULL                */
} EmuFilmRingResult;

size_t emu_film_ring_slot_bytes(void);
int emu_film_ring_create(int capacity, double idle_seconds, EmuFilmRing **out);
int emu_film_ring_submit(EmuFilmRing *ring, const EmuFilmRingRequest *req, long long *ticket);
int emu_film_ring_submit_many(EmuFilmRing *ring, const EmuFilmRingRequest *reqs, int n, long long *tickets,
                              int *n_submitted);
int emu_film_ring_poll(EmuFilmRing *ring, long long ticket, EmuFilmRingResult *out);
int emu_film_ring_poll_many(EmuFilmRing *ring, const long long *tickets, int n, const EmuFilmRingResult *outs,
                            int32_t *done);
int emu_film_ring_wait(EmuFilmRing *ring, long long ticket, double timeout_s, EmuFilmRingResult *out);
int emu_film_ring_ready(EmuFilmRing *ring, long long ticket);
int emu_film_ring_running(EmuFilmRing *ring);
int emu_film_ring_stop(EmuFilmRing *ring);
int emu_film_ring_destroy(EmuFilmRing *ring);

/* ------------------------------------------ dense linear algebra
 * Batched complex128 GEMM, C_b = alpha A_b B_b + beta C_b (row-major; A_b is
 * m x k, B_b k x n), and batched LU solve A_b X_b = B_b with partial pivoting
 * (A_b overwritten by its LU factors, B_b by X_b; ipiv 0-based; info[b] = 0
 * or j+1 for the first exactly-zero pivot).  These stand in for the
 * np.matrix products and np.linalg.solve (LAPACK zgesv) calls of
 * backend/stack.py:229-278 and backend/mode_calcs.py:498-513. */
int emu_zgemm_batched(int m, int n, int k, emu_c128 alpha, const emu_c128 *d_A, int lda,
                      long long stride_A, const emu_c128 *d_B, int ldb, long long stride_B,
                      emu_c128 beta, emu_c128 *d_C, int ldc, long long stride_C, int batch,
                      void *stream);
int emu_zgesv_batched(int n, int nrhs, emu_c128 *d_A, int lda, long long stride_A,
                      int32_t *d_ipiv, emu_c128 *d_B, int ldb, long long stride_B,
                      int32_t *d_info, int batch, void *stream);

/* ---------------------------------------------- a7: film interfaces
 * R12 = (Z2 - Z1)/(Z2 + Z1), T12 = 2 sqrt(Z2) sqrt(Z1)/(Z2 + Z1) for every
 * order and polarisation, Z from each film's sorted k_z, index n and the
 * normalised wavelength (R21 = -R12, T21 = T12).  Replaces r_t_mat_anallo
 * (backend/mode_calcs.py:451-477).  Outputs are the diagonals, [B][2 Npw]. */
int emu_film_interface_batch(int batch, int n_pw, const emu_c128 *d_kz1, const emu_c128 *d_n1,
                             const emu_c128 *d_kz2, const emu_c128 *d_n2,
                             const double *d_wl_norm, emu_c128 *d_R12, emu_c128 *d_T12,
                             void *stream);

/* ---------------------------------- a8: film / nanostructure interface
 * Batched r_t_mat_tf_ns (backend/mode_calcs.py:480-515): for each b,
 *   z = sqrt(1/Z_film), A = z o J, B = J_dag o z, S = I + B A,
 *   R12 = -I + 2 A S^-1 B (P x P), T12 = 2 S^-1 B (M x P),
 *   R21 = S^-1 (I - B A) (M x M), T21 = 2 A S^-1 (P x M),
 * with Z_film from the film's sorted k_z [b][P/2], index n [b] and
 * normalised wavelength [b] (backend/mode_calcs.py:199-218).
 * J [b][P][M] (already divided by the area ratio, mode_calcs.py:384-386),
 * J_dag [b][M][P].  info[b] != 0 marks an exactly singular I + B A. */
size_t emu_interface_dense_workspace_size(int batch, int P, int M);
int emu_interface_dense_batch(int batch, int P, int M, const emu_c128 *d_film_kz,
                              const emu_c128 *d_film_n, const double *d_wl_norm,
                              const emu_c128 *d_J, const emu_c128 *d_J_dag, emu_c128 *d_R12,
                              emu_c128 *d_T12, emu_c128 *d_R21, emu_c128 *d_T21,
                              int32_t *d_info, void *d_workspace, size_t workspace_bytes,
                              void *stream);

/* ------------------------------- a9, a10: dense cascade and fluxes
 * Net scattering matrices and energy fluxes of stacks with nanostructured
 * layers (backend/stack.py:162-426), one spectral point per batch item,
 * every item with the same layer shapes.  Layer i (bottom = 0) gives its
 * air-interface matrices: dense ones as R12 [P][P], T12 [M][P],
 * R21 [M][M], T21 [P][M]; film ones (dense = 0, M = P) as diagonals [P].
 * A zero stride shares a matrix across the batch. */
typedef struct {
  int M;                 /* modes of the layer (P for a film)               */
  int dense;             /* 1: dense interface matrices; 0: film diagonals  */
  const emu_c128 *d_R12, *d_T12, *d_R21, *d_T21;
  long long stride_R12, stride_T12, stride_R21, stride_T21; /* elements    */
  const emu_c128 *d_kz;  /* [b][M] k_z (finite layers)                      */
  long long stride_kz;
  double height_norm;    /* height / period (finite layers)                 */
  const double *d_height_norm; /* [b] per-point height / period, or NULL:
                                * height_norm for every point               */
} EmuLayer;

typedef struct {
  int batch, n_layers, P;
  const EmuLayer *h_layers;    /* host array [n_layers], bottom to top      */
  const double *h_shears;      /* host [n_layers][2] or NULL                */
  int shear_ncoord;            /* 1 or 2                                    */
  const double *d_air_alphas;  /* [batch][P/2] air alphas, unsorted         */
  const double *d_air_betas;   /* [batch][P/2] or NULL (1D)                 */
  int calc_fluxes;             /* needs a film superstrate                  */
  int pol;                     /* EMU_POL_*                                 */
  const emu_c128 *d_incoming;  /* [batch][P] for EMU_POL_INCOMING           */
  const int32_t *d_specular;   /* [batch] superstrate specular order        */
  const int32_t *d_num_prop;   /* [batch][3] propagating orders: air, superstrate, substrate */
  emu_c128 *d_R_net;           /* [batch][P][P]                             */
  emu_c128 *d_T_net;           /* [batch][M0][P]                            */
  double *d_fluxes;            /* [batch][L+1][2] or NULL: down fluxes (incoming, air gaps top
                                  to bottom, substrate) then the reflected flux */
  double *d_a_list, *d_t_list, *d_r_list; /* film substrate only, or NULL  */
  uint32_t *d_flags;           /* [batch] EMU_PT_* or NULL                  */
  int32_t *d_info;             /* [batch] 0 or the first singular solve     */
  emu_c128 *d_vec_coef_down;   /* [batch][stride] or NULL                   */
  emu_c128 *d_vec_coef_up;
  long long vec_coef_down_stride, vec_coef_up_stride;
  int save_lists;              /* 1: fill d_tnet_list / d_rnet_list         */
  emu_c128 *d_tnet_list;       /* [batch][2L-2][list_stride]                */
  emu_c128 *d_rnet_list;
  int mode;                    /* 0 auto; 1 one CTA per solve; 2 each step
                                  spread over many CTAs (large matrices, few
                                  solves); identical results                 */
} EmuStackDense;

size_t emu_stack_dense_workspace_size(const EmuStackDense *p);
long long emu_stack_dense_list_stride(const EmuStackDense *p);
int emu_stack_dense_batch(const EmuStackDense *p, void *d_workspace, size_t workspace_bytes,
                          void *stream);

/* ------------------- a9, a10: uneven batch of dense stacks, one launch
 * Stacks of different shapes -- plane-wave count P, layer count, Bloch-mode
 * counts, polarisation -- each the whole Stack.calc_scat of one spectral
 * point (backend/stack.py:162-426) with a film substrate and a film
 * superstrate, solved in ONE launch: a persistent kernel whose CTAs take
 * stacks in the given order (costliest first) from an atomic counter and
 * run the cascade and the flux pass of emu_stack_dense_batch's one-CTA path
 * (same arithmetic, same results).  Layer matrices are read where they lie
 * (any device pointers, e.g. a cache of layer interfaces); descriptors live
 * in device memory and are bounds-checked against the packed arrays: a bad
 * one marks its stack EMU_PT_BAD_POINT in d_flags and is skipped.
 * No counterpart call in the reference (it solves one Stack per call). */
typedef struct {
  int M, dense;                /* as EmuLayer (film: dense = 0, M = P)      */
  const emu_c128 *d_R12, *d_T12, *d_R21, *d_T21; /* this stack's matrices */
  const emu_c128 *d_kz;        /* [M] (finite layers)                       */
  double height_norm;          /* height / period (finite layers)           */
} EmuVarLayer;

typedef struct {
  int n_layers, P, pol, spec;  /* pol EMU_POL_*; spec: superstrate specular */
  int num_prop[3];             /* propagating orders: air, superstrate, substrate */
  int _pad;
  long long layer_off;         /* first of n_layers entries in d_layers     */
  long long inc_off;           /* [P] in d_incoming (EMU_POL_INCOMING)      */
  long long rnet_off;          /* [P][P] in d_R_net                         */
  long long tnet_off;          /* [P][P] in d_T_net                         */
  long long list_off;          /* [L-1] in d_a_list / d_t_list              */
  long long flux_off;          /* [L+1][2] in d_fluxes                      */
} EmuStackPoint;

typedef struct {
  int n_stacks;
  const EmuStackPoint *d_points;   /* [n_stacks]                            */
  const int32_t *d_order;          /* [n_stacks] processing order, or NULL  */
  const EmuVarLayer *d_layers;     /* packed layer descriptors              */
  long long n_layer_desc;          /* entries in d_layers                   */
  const emu_c128 *d_incoming;  long long incoming_len;
  emu_c128 *d_R_net;           long long rnet_len;
  emu_c128 *d_T_net;           long long tnet_len;
  double *d_a_list, *d_t_list; long long list_len;
  double *d_fluxes;            long long flux_len;   /* or NULL              */
  double *d_r_list;            /* [n_stacks]                                */
  uint32_t *d_flags;           /* [n_stacks] EMU_PT_*                       */
  int32_t *d_info;             /* [n_stacks] 0 or the first singular solve  */
  int max_P, max_D, max_L;     /* bounds of every stack: P, max(P, M), L    */
  int n_slots;                 /* CTAs (each with its own workspace); 0: as
                                  many as fit on the GPU at once             */
} EmuStackVarBatch;

/* Workspace for the batch: n_slots x the workspace of the largest stack.
 * emu_stack_var_slots gives the CTA count that n_slots = 0 selects. */
int emu_stack_var_slots(const EmuStackVarBatch *p);
size_t emu_stack_var_workspace_size(const EmuStackVarBatch *p);
int emu_stack_var_batch(const EmuStackVarBatch *p, void *d_workspace, size_t workspace_bytes,
                        void *stream);

/* ------------------------------------- a11, a12: overlap integrals
 * J (2 Npw x nval) and J_dag (nval x 2 Npw) of P2 Bloch-mode fields with the
 * TE ("E") and TM ("K") plane waves, by the 16-point triangle quadrature
 * over every element with the affine element map, rows in the sorted
 * plane-wave order (key -Re(kz^2), kz^2 = k0^2 - alpha^2 - beta^2).
 * Replaces J_overlap (backend/fortran/J_overlap.f:3-246, called from
 * backend/fortran/py_calc_modes.f:802-806), J_dagger_overlap
 * (backend/fortran/J_dagger_overlap.f:3-246, py_calc_modes.f:818-822),
 * pw_ordering (backend/fortran/pw_ordering.f:2-91) and the division
 * J / area_norm of backend/mode_calcs.py:384-386.
 * Fields use the reference layout sol(3, 13, nval, nel) (Fortran order),
 * i.e. [nel][nval][13][3] complex; table_nod is [nel][6], 1-based.
 * The plane-wave set is the caller's (emu_grating_orders), the set the
 * films of the same stack use. */
typedef struct {
  int batch;               /* problems (wavelengths) on one mesh            */
  int nval;                /* Bloch modes                                   */
  int nel, npt;            /* triangles, nodes                              */
  int n_pw;                /* plane waves per polarisation                  */
  int max_order;           /* max |px|, |py| of the order set (<= 24)       */
  const int32_t *d_px, *d_py; /* [Npw]                                      */
  const double *d_x;       /* [npt][2] coordinates in units of the period   */
  const int64_t *d_table_nod; /* [nel][6], 1-based                          */
  double d, dy;            /* lattice vectors (1, period_y/period)          */
  const double *d_bloch;   /* [batch][2] k_parallel * period                */
  const double *d_k0;      /* [batch] 2 pi / (wl / period)                  */
  const emu_c128 *d_sol1;  /* [batch][nel][nval][13][3] or NULL             */
  const emu_c128 *d_sol2;  /* adjoint fields, same layout, or NULL          */
  const emu_c128 *d_scale2;/* [batch][nval] normalisation of the adjoint modes or NULL */
  const int32_t *d_perm2;  /* [batch][nval] adjoint order after pair swaps or NULL */
  double area_norm;        /* period_y / period                             */
  emu_c128 *d_J;           /* [batch][2 Npw][nval] (with d_sol1)            */
  emu_c128 *d_J_dag;       /* [batch][nval][2 Npw] (with d_sol2)            */
  int32_t *d_index_pw_inv; /* [batch][Npw] 0-based sorted positions or NULL */
  int elements_per_chunk;  /* 0 = default (4096); bounds the workspace      */
  int precision;           /* 0: FP64 tensor-core GEMM (mma.sync f64); 1:
                              tcgen05 tensor cores, split-TF32 (hi + lo)
                              products, FP32 accumulation per 256 K values,
                              those chunk sums added in FP32 within a K split,
                              FP64 sum of the splits                          */
  int32_t *d_error;        /* [1] set to 1 if a bounded device wait gave up
                              (tensor-core path), else left untouched; may be NULL */
  int tc_splits;           /* tensor-core path: K splits per GEMM (1-256), 0 = one
                              wave of CTAs; never fewer than keep each split
                              within 32 chunks of 256 K values (each chunk is
                              accumulated apart: the tensor cores' FP32
                              accumulation drifts by ~7e-9 x K relative);
                              results differ by rounding between choices */
  int field_c64;           /* tensor-core path only: 1 = d_sol1 / d_sol2 hold
                              complex64 (float re, im) in the same layout (the
                              operands are FP32 anyway; half the bytes read) */
} EmuOverlap;

size_t emu_overlap_workspace_size(const EmuOverlap *p);
int emu_overlap_batch(const EmuOverlap *p, void *d_workspace, size_t workspace_bytes, void *stream);

/* ---------------------------------------- a13: Bloch-mode normalisation
 * Diagonal of the adjoint x prime orthogonality matrix
 *   ovl(n, n) = sum_el sol2_el(:, n)^T  M_el  (beta1(n) sol1_el(:, n)),
 * M_el the 12 x 22 P2-mass / P3-gradient element matrix times
 * pp(type_el) / k0 (backend/fortran/orthogonal.f:84-248), and the
 * normalisation factors scale(n) = 1 / sqrt(ovl(n, n))^2, or 1 when
 * |sqrt(ovl(n, n))| <= 1e-8 (backend/fortran/normalisation.f:15-31).
 * n_small[b] counts |ovl(n, n)| <= 1e-7, the trigger of the reference's
 * conjugate-pair reordering (orthogonal.f:252-301); the caller runs that
 * reordering (emu_mode_overlap_matrix gives the full matrix it needs). */
typedef struct {
  int batch, nval, nel, npt;
  const double *d_x;       /* [npt][2]                                      */
  const int64_t *d_table_nod; /* [nel][6], 1-based                          */
  const int64_t *d_type_el;/* [nel], 1-based                                */
  const emu_c128 *d_pp;    /* [n_types] (1 for the E-field formulation)     */
  const double *d_k0;      /* [batch]                                       */
  const emu_c128 *d_beta1; /* [batch][nval] prime propagation constants     */
  const emu_c128 *d_sol1, *d_sol2; /* [batch][nel][nval][13][3]             */
  emu_c128 *d_diag;        /* [batch][nval]                                 */
  emu_c128 *d_scale;       /* [batch][nval]                                 */
  int32_t *d_n_small;      /* [batch]                                       */
} EmuNormalise;

size_t emu_mode_overlap_workspace_size(const EmuNormalise *p);
int emu_mode_overlap_diag(const EmuNormalise *p, void *d_workspace, size_t workspace_bytes,
                          void *stream);

/* The conjugate-pair reordering of the adjoint modes
 * (backend/fortran/orthogonal.f:252-301), for problems whose diagonal has
 * entries |ovl(j, j)| <= 1e-7: computes the full matrix, runs the reference's
 * swap loop (each such adjoint mode j, unless it is the second of a pair just
 * handled, is exchanged with every later mode j2 with |ovl(j2, j)| > 1e-7),
 * and writes perm[b][i] (adjoint mode now at position i, to pass as
 * EmuOverlap.d_perm2), the recomputed diagonal ovl(perm[i], i) to d_diag,
 * its normalisation factors to d_scale and the reference's pair-warning
 * count to warn[b]. */
size_t emu_mode_overlap_reorder_workspace_size(const EmuNormalise *p);
int emu_mode_overlap_reorder(const EmuNormalise *p, int32_t *d_perm, int32_t *d_warn,
                             void *d_workspace, size_t workspace_bytes, void *stream);

/* ----------------------------- a11, a12 for 1D gratings ('1D_array')
 * Plane-wave order of the 1D set px = -max_order..max_order: the rank of
 * each order (generation index s = px + max_order) when the keys
 * -Re(kz^2), kz = sqrt(k0^2 - alpha^2 - beta^2), alpha = bloch_x +
 * 2 pi px / period_x, beta = bloch_y, are sorted by the reference's
 * quicksort (ties ranked as it ranks them).  Replaces pw_ordering_1d
 * (backend/fortran/pw_ordering_1d.f:1-80 with z_indexx.f).  Host only.
 * h_index_pw_inv: [2 max_order + 1], 0-based. */
int emu_pw_order_1d(int max_order, double period_x, double bloch_x, double bloch_y, double k0,
                    int32_t *h_index_pw_inv);

/* Row of each 1D order (generation index) in the 2D order set of the same
 * max_order built with period_x in both directions, sorted the same way:
 * the placement of pw_matrix_1d_to_2d (backend/fortran/pw_matrix_1d_to_2d.f:
 * 60-120).  Host only.  h_row_2d may be NULL to query *h_npw_2d (the 2D
 * set's size); capacity >= 2 max_order + 1 otherwise. */
int emu_pw_embed_1d_to_2d(int max_order, double period_x, double bloch_x, double bloch_y,
                          double k0, int32_t *h_row_2d, int capacity, int *h_npw_2d);

/* J (2 Npw x nval: E rows then K rows) and J_dag (nval x 2 Npw) of 1D
 * Bloch-mode fields with the plane waves exp(-i alpha x) and exp(+i alpha x)
 * (Npw = 2 max_order + 1), rows at the sorted positions of
 * emu_pw_order_1d; with d_row_2d also both matrices embedded in the 2D
 * order set (zero outside the (px, 0) rows).  Replaces J_overlap_1d
 * (backend/fortran/J_overlap_1d.f:8-225), J_dagger_overlap_1d
 * (backend/fortran/J_dagger_overlap_1d.f:1-225) and pw_matrix_1d_to_2d,
 * called from backend/fortran/py_calc_modes_1d.f:583-620 and returned by
 * backend/mode_calcs.py:323-355 (J, J_dag when world_1d, else J_2d,
 * J_dag_2d; no area division for 1D layers).
 * Fields use the reference layout sol(11, nval, nel) (Fortran order), i.e.
 * [nel][nval][11] complex: Ex at the P2 nodes (x_min, x_max, midpoint), Ey
 * at the P3 nodes (x_min, x_max, x_min + h/3, x_min + 2h/3), Ez (unused);
 * table_nod is [nel][3], 1-based, its first two entries the element's end
 * nodes.  An element whose end nodes fall outside [1, npt] is skipped and
 * *d_error set to 1. */
typedef struct {
  int batch;               /* problems (wavelengths / k_parallel) on one mesh */
  int nval;                /* Bloch modes                                   */
  int nel, npt;            /* elements, P2 nodes                            */
  int max_order;           /* 1D orders px = -max_order..max_order          */
  const double *d_x;       /* [npt] node coordinates                        */
  const int64_t *d_table_nod; /* [nel][3], 1-based                          */
  double period_x;         /* period in the units of d_x (the reference's
                              period_x: the span of the periodic nodes)     */
  const double *d_bloch;   /* [batch][2] bloch_vec_x, bloch_vec_y           */
  const int32_t *d_index_pw_inv; /* [batch][Npw] from emu_pw_order_1d       */
  const emu_c128 *d_sol1;  /* [batch][nel][nval][11] or NULL                */
  const emu_c128 *d_sol2;  /* adjoint fields, same layout, or NULL          */
  const emu_c128 *d_scale; /* [batch][nval] normalisation of prime and adjoint
                              mode n (emu_mode_overlap_1d), or NULL         */
  const int32_t *d_perm2;  /* [batch][nval] adjoint mode taken for mode n
                              after conjugate-pair swaps, or NULL           */
  emu_c128 *d_J;           /* [batch][2 Npw][nval] (with d_sol1)            */
  emu_c128 *d_J_dag;       /* [batch][nval][2 Npw] (with d_sol2)            */
  int npw_2d;              /* 2D embedding: the 2D set's size, or 0         */
  const int32_t *d_row_2d; /* [batch][Npw] from emu_pw_embed_1d_to_2d, or NULL */
  emu_c128 *d_J_2d;        /* [batch][2 npw_2d][nval]                       */
  emu_c128 *d_J_dag_2d;    /* [batch][nval][2 npw_2d]                       */
  int32_t *d_error;        /* [1] or NULL                                   */
} EmuOverlap1D;

int emu_overlap1d_batch(const EmuOverlap1D *p, void *stream);

/* Orthogonality of the adjoint and prime 1D Bloch modes,
 *   <i|j> = beta1(j) / k0 sum_el pp(type) (u_x Mxx v_x + u_y Myy v_y
 *           - u_x Kxy v_z - i bloch_y u_y Myy v_z),
 * u the adjoint mode perm2[i] and v the prime mode j on each element
 * (Mxx, Myy the P2 and P3 mass matrices, Kxy = int phi_P2 dpsi_P3/dx).
 * full = 0: the diagonal into d_out [batch][nval], the normalisation
 * factors 1/sqrt(<m|m>) (1 where |sqrt| <= 1e-8) into d_scale (optional)
 * and the count of |<m|m>| <= 1e-7 into d_n_small (optional); full = 1: the
 * whole matrix into d_out [batch][nval][nval].  Replaces orthogonal_1d
 * (backend/fortran/orthogonal_1d.f:1-158; its conjugate-pair swap loop,
 * :160-215, runs on the host over the full matrix) and normalisation_1d
 * (backend/fortran/normalisation_1d.f:1-34), called from
 * backend/fortran/py_calc_modes_1d.f:531-547. */
typedef struct {
  int batch, nval, nel, npt;
  int n_types;               /* material types (1-based in d_type_el)       */
  const double *d_x;         /* [npt]                                       */
  const int64_t *d_table_nod;/* [nel][3], 1-based                           */
  const int64_t *d_type_el;  /* [nel], 1-based                              */
  const emu_c128 *d_pp;      /* [n_types]                                   */
  const double *d_k0;        /* [batch] 2 pi / wl_norm                      */
  const double *d_bloch;     /* [batch][2]                                  */
  const emu_c128 *d_beta1;   /* [batch][nval] prime propagation constants   */
  const emu_c128 *d_sol1;    /* [batch][nel][nval][11]                      */
  const emu_c128 *d_sol2;    /* [batch][nel][nval][11]                      */
  const int32_t *d_perm2;    /* [batch][nval] or NULL                       */
  emu_c128 *d_out;
  emu_c128 *d_scale;         /* [batch][nval] or NULL                       */
  int32_t *d_n_small;        /* [batch] or NULL                             */
  int32_t *d_error;          /* [1] or NULL                                 */
} EmuNormalise1D;

int emu_mode_overlap_1d(const EmuNormalise1D *p, int full, void *stream);

/* Allocation-free variant of emu_film_stack_batch (no counterpart in the
 * reference, which has no GPU path).  For callers that cannot allocate
 * device memory where they solve -- a thread in a latency-critical loop
 * (cudaMalloc / cudaFree synchronise the device), code running while
 * another framework's caching allocator owns the device heap, or an
 * embedding that must not fail on memory pressure after start-up -- the
 * solve uses a scratch array of emu_film_stack_static_scratch_bytes()
 * (16 MiB) compiled into the library instead of a caller workspace.  The
 * caller still passes every input and output buffer.
 *   - Only incoming amplitudes (EMU_POL_INCOMING) use the array; requests
 *     whose emu_film_stack_workspace_size() exceeds its size (about 8 700
 *     points x orders of a 12-layer stack, e.g. 107 points at Npw = 81) are
 *     rejected with EMU_E_WORKSPACE (split the batch).  The standard
 *     polarisations use no scratch and have no size limit here.
 *   - The first call on a device looks up that device's copy of the array
 *     (cudaGetSymbolAddress); make that first call before any stream
 *     capture.
 *   - All calls share the one array per device: calls that can overlap on
 *     the GPU (different streams, other host threads) race on it; order
 *     them on one stream.  Nothing in it needs to start at zero.
 *   - No cudaMalloc, cudaFree or allocating library routine is called. */
size_t emu_film_stack_static_scratch_bytes(void);
int emu_film_stack_batch_noalloc(const EmuFilmStackBatch *p, void *stream);

/* --------------------------------- a2-a4, a7, a9, a10: uneven film batches
 * The film solve of emu_film_stack_batch for a batch whose points differ in
 * shape: each point brings its own layer count, order set (Npw, 1D or 2D),
 * periods, polarisation, wavelength and k_parallel -- in the reference, one
 * Stack(layers).calc_scat(pol) call each (backend/stack.py:162-426), made in
 * a loop or a process pool over wavelengths and structures.  One warp
 * solves one point; points of any mix of shapes share one launch.
 *
 * Every per-point array is packed: the point's slices start at its offsets
 * (counted in elements of the array they index).  Offsets and sizes come
 * from emu_film_var_plan, which also sizes the workspace.  Outputs match
 * emu_film_stack_batch's for the same point (sorted-order R_net / T_net
 * diagonals, a_list / t_list / r_list, EMU_PT_* flags).  A point whose
 * descriptor is out of range (L < 2, Npw < 1, L or Npw above the batch
 * bounds, bad pol, a slice outside its array) is not solved and gets
 * EMU_PT_BAD_POINT. */
#define EMU_PT_BAD_POINT 32u     /* descriptor out of range: point skipped  */

typedef struct {
  int32_t n_layers;      /* L >= 2                                          */
  int32_t n_pw;          /* Npw of this point's order set                   */
  int32_t world_1d;
  int32_t pol;           /* EMU_POL_*                                       */
  int64_t order_off;     /* d_px / d_py: Npw orders (emu_grating_orders)    */
  int64_t n_off;         /* d_n: L indices, substrate first                 */
  int64_t h_off;         /* d_heights_nm: L-2 heights                       */
  int64_t inc_off;       /* d_incoming: 2 Npw (pol == EMU_POL_INCOMING)     */
  int64_t rt_off;        /* d_R_net / d_T_net: 2 Npw        (set by plan)   */
  int64_t list_off;      /* d_a_list / d_t_list: L-1        (set by plan)   */
  int64_t np_off;        /* d_num_prop: L+1                 (set by plan)   */
  int64_t ws_off;        /* workspace, bytes                (set by plan)   */
  double period, period_y; /* nm                                            */
  double wl_nm;          /* wavelength (nm)                                 */
  double kx, ky;         /* k_parallel (nm^-1)                              */
} EmuFilmPoint;

typedef struct {
  int n_points;                /* B                                         */
  int max_layers, max_pw;      /* bounds over the points (from the plan)    */
  const EmuFilmPoint *d_points;/* [B]                                       */
  const int32_t *d_order;      /* [B] solve order (costliest first) or NULL */
  const int32_t *d_px, *d_py;
  const emu_c128 *d_n;
  const double *d_heights_nm;
  const emu_c128 *d_incoming;  /* NULL unless some pol == EMU_POL_INCOMING  */
  emu_c128 *d_R_net, *d_T_net; /* sum of 2 Npw                              */
  double *d_a_list, *d_t_list; /* sum of L-1                                */
  double *d_r_list;            /* [B]                                       */
  uint32_t *d_flags;           /* [B]                                       */
  int32_t *d_specular;         /* [B] or NULL                               */
  int32_t *d_num_prop;         /* sum of L+1 or NULL                        */
  /* lengths (elements) of the packed arrays above: a point whose slices
   * fall outside them, or outside the workspace, gets EMU_PT_BAD_POINT */
  int64_t order_len, n_len, h_len, inc_len, rt_len, list_len, np_len;
  int warps_per_cta;           /* 1-8 warps (points) per CTA, 0 = 8 (fewer if
                                  the shared-memory slots do not fit); speed only */
  int variant;                 /* register budget: 0 = 2 CTAs per SM (128
                                  registers), 1 = 3 (85); speed only */
} EmuFilmVarBatch;

/* Host-side plan over the host copy of the descriptors: fills rt_off,
 * list_off, np_off and ws_off, returns the output lengths (elements) and
 * the workspace bytes, the bounds for max_layers / max_pw, and (when
 * h_order is not NULL) a costliest-first solve order.  Returns EMU_E_SHAPE
 * for a point out of range. */
int emu_film_var_plan(EmuFilmPoint *h_points, int n_points, int32_t *h_order,
                      int64_t *rt_len, int64_t *list_len, int64_t *np_len,
                      size_t *workspace_bytes, int *max_layers, int *max_pw);
int emu_film_var_batch(const EmuFilmVarBatch *p, void *d_workspace, size_t workspace_bytes,
                       void *stream);

/* Tensor-core GEMM used by the overlap integrals, exposed for testing:
 * C (m x n, FP64) = A (m x k) . B (n x k)^T with both operands split into
 * TF32 hi + lo parts, three tcgen05 MMAs per step (hi.hi + hi.lo + lo.hi),
 * FP32 accumulation in tensor memory over each of `splits` K ranges and an
 * FP64 sum of the ranges.  d_err[0] is set to 1 if a bounded device wait
 * gave up.  No counterpart in the reference (which has no GPU path); it
 * stands in for the FP64 contraction of J_overlap.f:162-184. */
size_t emu_tc_gemm_workspace_size(int m, int n, int k, int splits);
int emu_tc_gemm_tf32x3(int m, int n, int k, const double *d_A, const double *d_B, double *d_C,
                       int splits, int32_t *d_err, void *d_workspace, size_t workspace_bytes,
                       void *stream);

/* ------------------------------------------------------- measurement
 * FP64 FMA throughput probe: blocks x threads threads each run 64 dependent
 * FMA chains of `iters` steps (2*64*iters*threads*blocks flops).  Used as the
 * FP64 roofline denominator of the film kernels; the reference has no
 * counterpart (it has no GPU path). */
int emu_probe_fp64(int blocks, int threads, int iters, double *d_out, void *stream);

/* ------------------------------------- f1: FEM Bloch modes of a 2D layer
 * The mode solve of calc_modes_2d (backend/fortran/py_calc_modes.f:243-700)
 * for the E-field formulation with periodic boundaries, as the reference
 * runs it (backend/mode_calcs.py:268-381): the mixed element of asmbly.f
 * (per triangle a face and 3 edges with 3 transverse DOFs each, basis of
 * basis_ls.f / basis_vec.f, and 10 P3 nodes with one E_z DOF), Bloch phase
 * factors on periodic images, the generalised problem K x = beta^2 M x
 * solved by shift and invert, and the nodal fields of array_sol.f.
 *
 * emu_fem_topology (host): pairs the periodic boundary nodes as
 * periodic_node.f does (lowest index of a class is its origin; pairs differ
 * by a lattice vector ix a1 + iy a2, |ix|, |iy| <= 1, within 1e-6 in the
 * 1-norm), numbers the DOFs (an entity and its periodic images share
 * them), and builds the CSR pattern of K and M (row = trial DOF, column =
 * test DOF, columns ascending) with, for every CSR entry, the element-matrix
 * entries it sums in element order (src: flat indices e*484 + a*22 + b).
 * Outputs are caller-allocated to the bounds given; neq and nnz are set.
 * Returns EMU_E_ARG for a boundary node without a periodic image or an edge
 * whose ends are images of each other. */
typedef struct {
  int npt, nel;
  const double *h_x;          /* [npt][2], the unit cell in units of the period */
  const int32_t *h_type_nod;  /* [npt], non-zero on the cell boundary           */
  const int64_t *h_table_nod; /* [nel][6], 1-based (vertices, then mid-edge
                                 nodes of edges 1-2, 2-3, 1-3)                  */
  int32_t *h_dof;             /* out [nel][22]: 12 transverse, 10 E_z           */
  double *h_shift;            /* out [nel][14][2]: lattice shift of each entity
                                 instance (face, 3 edges, 10 P3 nodes)          */
  int8_t *h_ends;             /* out [nel][3][2]: local vertices of each edge,
                                 the lower mapped node number first             */
  int32_t *h_row_ptr;         /* out [neq + 1], bound nel*22 + 1                */
  int32_t *h_col;             /* out [nnz], bound nel*484                       */
  int32_t *h_src_ptr;         /* out [nnz + 1], bound nel*484 + 1               */
  int32_t *h_src;             /* out [nel*484]                                  */
  int neq, nnz;               /* out */
} EmuFemTopology;

int emu_fem_topology(EmuFemTopology *t);

/* Element matrices K_e, M_e [nel][22][22] (trial row, test column) of
 * asmbly.f:130-320 with pp = 1, qq = n^2 k0^2 per material type, each entry
 * times val_exp(test) conj(val_exp(trial)), val_exp = exp(i bloch . shift),
 * 16-point rule (quad_triangle.f), affine element maps (curved_elem_tri.f
 * makes every element straight).  n_types <= 8. */
typedef struct {
  int nel, n_types;
  const double *d_x;            /* [npt][2]                     */
  const int64_t *d_table_nod;   /* [nel][6], 1-based            */
  const int64_t *d_type_el;     /* [nel], 1-based               */
  const double *d_shift;        /* [nel][14][2] (emu_fem_topology) */
  const int8_t *d_ends;         /* [nel][3][2]                  */
  emu_c128 n_eff[8];            /* index of each material type  */
  double k0;                    /* 2 pi / (wl / period)         */
  double bloch[2];              /* k_parallel * period          */
  emu_c128 *d_Ke, *d_Me;        /* out [nel][22][22]            */
} EmuFemElements;

int emu_fem_element_matrices(const EmuFemElements *p, void *stream);

/* Global K, M values on the CSR pattern: each entry the sum of its element
 * entries in element order (deterministic).  Then, optionally, the dense
 * shifted matrix A = K - shift M (row-major n x n, lda >= n; every other
 * entry set to zero), which emu_fem_lu factors in place (partial pivoting;
 * panels of the dense interface path's LU inside outer blocks of 256
 * columns; ipiv 0-based, info 0 or the first zero pivot + 1) and
 * emu_fem_inverse turns into the columns d_cols of A^-1 (a separate
 * [n][ldi] buffer; d_cols NULL with ncols = n for all of A^-1). */
int emu_fem_assemble(int nnz, const int32_t *d_src_ptr, const int32_t *d_src, const emu_c128 *d_Ke,
                     const emu_c128 *d_Me, emu_c128 *d_K, emu_c128 *d_M, void *stream);
int emu_fem_shifted_dense(int neq, const int32_t *d_row_ptr, const int32_t *d_col, const emu_c128 *d_K,
                          const emu_c128 *d_M, emu_c128 shift, emu_c128 *d_A, int lda, void *stream);
int emu_fem_lu(int n, emu_c128 *d_A, int lda, int32_t *d_ipiv, int32_t *d_info, void *stream);
int emu_fem_inverse(int n, const emu_c128 *d_LU, int lda, const int32_t *d_ipiv, int ncols,
                    const int32_t *d_cols, emu_c128 *d_Ainv, int ldi, void *stream);

/* Y = (K - shift M)^-1 M X for a block of nrhs vectors (X [n][ldx], Y
 * [n][ldy], row-major, vector r in column r; T [ncols][nrhs] scratch): the
 * operator of the shift-and-invert eigen-solve (valpr_umf_64.f:314-383,
 * which applies it one vector at a time through UMFPACK's solves), here a
 * sparse product with M on the rows d_cols where M has entries (the
 * transverse DOFs; NULL with ncols = n for all rows) and one pass over
 * the matching columns of A^-1 ([n][ldi], from emu_fem_inverse with the same
 * d_cols) per 16 vectors. */
int emu_fem_apply_op(int n, int nrhs, const emu_c128 *d_Ainv, int ldi, int ncols, const int32_t *d_cols,
                     const int32_t *d_row_ptr, const int32_t *d_col, const emu_c128 *d_M, const emu_c128 *d_X,
                     int ldx, emu_c128 *d_T, emu_c128 *d_Y, int ldy, void *stream);

/* Nodal fields of array_sol.f:88-300: sol [nel][nval][13][3] (E_x, E_y,
 * E_z at the six P2 nodes, E_z interpolated from the P3 values; E_z at P3
 * nodes 4-10 in entries 6-12) from eigenvectors vec [neq][ldv] (mode m in
 * column m, already in output order), each mode divided by its first
 * largest-modulus P2-node component (elements, then nodes, then
 * components).  Workspace: emu_fem_fields_workspace_size. */
typedef struct {
  int nel, neq, nval;
  const double *d_x;
  const int64_t *d_table_nod;
  const double *d_shift;
  const int8_t *d_ends;
  const int32_t *d_dof;
  double bloch[2];
  const emu_c128 *d_vec;
  int ldv;
  emu_c128 *d_sol;              /* out [nel][nval][13][3] */
} EmuFemFields;

/* Order of the modes (host): z_indexx.f on the key -Re(beta^2) as
 * py_calc_modes.f:683 ranks them, ties where that quicksort puts them;
 * h_index 0-based. */
int emu_fem_mode_order(int n, const emu_c128 *h_beta, int32_t *h_index);

size_t emu_fem_fields_workspace_size(const EmuFemFields *p);
int emu_fem_nodal_fields(const EmuFemFields *p, void *d_workspace, size_t workspace_bytes, void *stream);

/* ------------------------------- f1: FEM Bloch modes of a 1D grating
 * The mode solve of calc_modes_1d (backend/fortran/py_calc_modes_1d.f:
 * 330-500, as backend/mode_calcs.py:323-341 calls it): E_x on discontinuous
 * P2 elements, E_y and E_z on continuous P3 elements, periodic
 * (periodic_cond_1d.f); element matrices of asmbly_1d.f; then the same
 * emu_fem_assemble / _shifted_dense / _lu / _inverse / _apply_op as the 2D
 * solve (11 local DOFs instead of 22) and emu_fem_mode_order.
 *
 * emu_fem1d_topology (host): elements must run left to right without gaps
 * (table_nod: x_min node, x_max node, middle node); equations numbered
 * element by element (E_x 3, then E_y and E_z at x_min, h/3, 2h/3), the last
 * element's x_max values sharing the first element's x_min equations with
 * the Bloch phase of one period.  Outputs caller-allocated to the bounds
 * given; neq (= 9 nel), nnz and the period are set.  EMU_E_ARG for
 * out-of-range nodes or unordered elements. */
typedef struct {
  int npt, nel;
  const double *h_x;           /* [npt] P2 node coordinates                      */
  const int64_t *h_table_nod;  /* [nel][3], 1-based                              */
  int32_t *h_dof;              /* out [nel][11]: E_x (3), E_y (4), E_z (4)       */
  double *h_shift;             /* out [nel][11]: the period for the last
                                  element's x_max values, else 0                 */
  int32_t *h_row_ptr;          /* out [neq + 1], bound 9 nel + 1                 */
  int32_t *h_col;              /* out [nnz], bound 121 nel                       */
  int32_t *h_src_ptr;          /* out [nnz + 1], bound 121 nel + 1               */
  int32_t *h_src;              /* out [121 nel]                                  */
  int neq, nnz;                /* out */
  double period;               /* out: span of the cell                          */
} EmuFem1dTopology;

int emu_fem1d_topology(EmuFem1dTopology *t);

/* Element matrices K_e, M_e [nel][11][11] (trial row, test column) of
 * asmbly_1d.f:150-250 with pp = 1, qq = n^2 k0^2, the reference element's
 * integrals of matrix_*_1d.f, each entry times val_exp(test)
 * conj(val_exp(trial)), val_exp = exp(i bloch_x shift). */
typedef struct {
  int nel, n_types;
  const double *d_x;            /* [npt]                 */
  const int64_t *d_table_nod;   /* [nel][3], 1-based     */
  const int64_t *d_type_el;     /* [nel], 1-based        */
  const double *d_shift;        /* [nel][11]             */
  emu_c128 n_eff[8];
  double k0;                    /* 2 pi / (wl / period)  */
  double bloch[2];              /* k_parallel * period   */
  emu_c128 *d_Ke, *d_Me;        /* out [nel][11][11]     */
} EmuFem1dElements;

int emu_fem1d_element_matrices(const EmuFem1dElements *p, void *stream);

/* Nodal values of array_sol_1d.f:60-220: sol [nel][nval][11] from
 * eigenvectors vec [neq][ldv] (mode m in column m, in output order), each
 * mode divided by its first largest value within a quarter element of the
 * cell's middle when that is at least 0.95 of its first largest value,
 * else by its first largest value right of the middle (adjoint = 0, prime
 * modes) or left of it (adjoint = 1). */
typedef struct {
  int nel, neq, nval;
  const double *d_x;
  const int64_t *d_table_nod;
  const double *d_shift;
  const int32_t *d_dof;
  double bloch_x;
  int adjoint;
  const emu_c128 *d_vec;
  int ldv;
  emu_c128 *d_sol;              /* out [nel][nval][11] */
} EmuFem1dFields;

size_t emu_fem1d_fields_workspace_size(const EmuFem1dFields *p);
int emu_fem1d_nodal_fields(const EmuFem1dFields *p, void *d_workspace, size_t workspace_bytes, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* EMUSTACK_GSM_H */
