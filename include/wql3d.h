/*
 * wql3d.h -- C ABI of the B200-native WaveQLab3D per-step volume update.
 *
 * One library (libwql3d.so, sm_100a) advances one or two structured blocks of
 * the elastic / anelastic wave equation with the 6th-order traditional SBP
 * operator, SAT boundary and interface closures, compact ADE-PML, Q4 / Q8 /
 * fQ8 memory variables, moment-tensor point sources and the
 * Kennedy-Carpenter (5,4) low-storage Runge-Kutta scheme.
 *
 * The entry points are the seams of the reference Fortran driver
 * (paths relative to the reference project root):
 *   - domain stage ops   src/domain.f90:615-1017  (scale_rates, set_rates,
 *                         enforce_bound_iface_conditions, update_fields)
 *   - time step          src/time_step.f90:68-150 (time_step_RK)
 *   - rk vector backend  src/rk_vector_cpu.f90:7-18, src/rk_vector_openacc.f90:8-75
 *                         (scale_rate_array, update_state_array)
 *   - RHS backend        src/traditional_cartesian_rhs_cpu.f90:8-15
 *                         (try_traditional_cartesian_rhs)
 *   - final diagnostics  src/domain.f90:505-613 (close_domain)
 *
 * Conventions
 *   - Every function returns 0 on success or a negative WQL3D_E* code and
 *     never exits the process; wql3d_last_error() describes the last failure
 *     of the calling thread.
 *   - Host arrays are Fortran ordered (q/x fastest).  Each 3-D component
 *     covers (1-host_nb : n+host_nb) per axis, so a Fortran array allocated by
 *     allocate_array_body with ghost_nodes (nb = 3) is passed with host_nb = 3
 *     and an interior-only array with host_nb = 0.  Components follow one
 *     another (the 4th Fortran index is slowest).
 *   - Field order is v_x, v_y, v_z, s_xx, s_yy, s_zz, s_xy, s_xz, s_yz
 *     (src/JU_xJU_yJU_z6.f90:8-10).
 *   - One domain owns one CUDA stream; calls on one domain are not
 *     reentrant.  Domains are independent.
 */
#ifndef WQL3D_H
#define WQL3D_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WQL3D_ABI_VERSION 4

/* status codes */
#define WQL3D_OK 0
#define WQL3D_EINVAL (-1)       /* bad argument or unsupported combination */
#define WQL3D_ECUDA (-2)        /* CUDA runtime error */
#define WQL3D_ENOMEM (-3)       /* device allocation failed */
#define WQL3D_ENONFINITE (-4)   /* non-finite state detected (RUN-ELASTIC-001 family) */
#define WQL3D_ESTATE (-5)       /* call out of order */

/* mesh kinds (type_of_mesh) */
#define WQL3D_MESH_CARTESIAN 0
#define WQL3D_MESH_CURVILINEAR 1

/* derivative operator (fd_type / order of &problem_list) */
#define WQL3D_FD_TRADITIONAL6 0       /* traditional 6th-order SBP, src/JU_xJU_yJU_z6.f90:12-809, :16088-16640 */
#define WQL3D_FD_UPWIND4 1            /* upwind 4th order: forward operator on velocities, backward on stresses,
                                         src/JU_xJU_yJU_z6.f90:1439-2033, :17865-18400 (SAT tau0 = 144/49) */
#define WQL3D_FD_UPWIND6 2            /* upwind 6th order, src/JU_xJU_yJU_z6.f90:2665-3688, :18958-19510
                                         (tau0 = 42300/13613) */
#define WQL3D_FD_UPWIND_DRP6 3        /* upwind DRP 6th order, src/JU_xJU_yJU_z6.f90:10556-12058 and
                                         JJU_x6_interior_upwind_drp (tau0 = 3.39644507697204) */

/* arithmetic */
#define WQL3D_FP64 0
#define WQL3D_FP32_COMPENSATED 1

/* response */
#define WQL3D_ELASTIC 0
#define WQL3D_Q4 1
#define WQL3D_Q8 2
#define WQL3D_FQ8 3

/* interface coupling (src/Interface_Condition.f90:348-378) */
#define WQL3D_IFACE_LOCKED 0
#define WQL3D_IFACE_SLIP_WEAKENING 1
#define WQL3D_IFACE_LINEAR 2
#define WQL3D_IFACE_RATE_STATE 3      /* rate-and-state, Regula-Falsi slip rate (src/Interface_Condition.f90:918-1263) */

/* fault prestress and static friction: per-point maps (iface_tau0, iface_fs)
   or the reference's TPV5 formulas (src/Interface_Condition.f90:1283-1294,
   1822-1830) evaluated at the face coordinates */
#define WQL3D_FAULT_MAPS 0
#define WQL3D_FAULT_TPV5 1
#define WQL3D_FAULT_TPV101 2          /* rate-and-state TPV101 / TPV102 prestress and parameters */
#define WQL3D_FAULT_TPV102 3
#define WQL3D_FAULT_TPV28 4           /* slip-weakening TPV28: fault_stress projected on each fault point's
                                         (n, m, l) basis plus the nucleation shear, fs / fd / Dc of
                                         src/Interface_Condition.f90:1459-1474, 2049-2076 */

/* fault outputs of wql3d_get_fault_output (src/domain.f90:782-845,
   src/fault_output.f90:73-122): [component][ns][nr] doubles */
#define WQL3D_FO_S 0       /* 4: slip along n, m, l and cumulative |slip rate| integral */
#define WQL3D_FO_SVEL 1    /* 3: v_hat - u_hat in (n, m, l), recorded at stage 1 */
#define WQL3D_FO_UHAT 2    /* 6: slip velocity (3) and side-1 traction + prestress (3), stage 1 */
#define WQL3D_FO_VHAT 3    /* 6: slip velocity (3) and side-2 traction + prestress (3), stage 1 */
#define WQL3D_FO_STATE 4   /* 1: state variable W */
#define WQL3D_FO_TRUP 5    /* 1: rupture time (1e9 where the slip rate never exceeded 1e-3) */

typedef struct wql3d_domain wql3d_domain;

/* Per-block description, filled once from the resolved configuration
   (src/block.f90:31-320 init_block). */
typedef struct wql3d_block_desc {
  int32_t nq, nr, ns;          /* grid points per axis */
  int32_t mesh;                /* WQL3D_MESH_* */
  int32_t f32_literal;         /* 1: SBP row-4 literal 0.013435342414630 in single precision
                                  (reference built without -r8 / -fdefault-real-8) */
  int32_t bc[6];               /* type_of_bc on faces Lx,Rx,Ly,Ry,Lz,Rz: 1 absorbing,
                                  2 free surface, 3 clamped, 0 interface, -1 none */
  int32_t pml[6];              /* PML slab per face (1..6 = Lx,Rx,Ly,Ry,Lz,Rz) */
  int32_t npml;                /* PML thickness in points */
  double aqrs[3], bqrs[3];     /* Cartesian block extents (mesh_source = 'compute') */
  double tau0;                 /* SAT penalty, 1/0.315949074074074 for traditional-6 */
  int32_t host_nb;             /* ghost width of the host arrays below */
  const double *coords;        /* curvilinear: 3 components x, y, z; NULL for Cartesian */
  const double *material;      /* 3 components lambda, mu, rho (already modulus-corrected) */
  const double *qs_inv;        /* Q4/Q8: 1/Qs per point (NULL: use Qs0 below) */
  const double *qp_inv;        /* Q4/Q8: 1/Qp per point */
  /* moment-tensor sources, src/moment_tensor.f90:8-740 */
  int32_t nsrc;
  int32_t src_order;           /* 2: 5-point delta, 4: 9-point delta */
  int32_t src_alpha;           /* 0, 25, 50 or 100 (order 4 weights) */
  const int32_t *src_type;     /* per source: 0 gaussian, 1 LOH_discontinuity, 2 Brune, 3 Cos-Bell,
                                  4 cosine, 5 LOH_moment_time_history, 6 sine_moment_time_history,
                                  7 ricker (f0 = duration, delay = t_init) */
  const double *src_par;       /* per source 11 values: duration t_init mxx myy mzz mxy mxz myz x y z */
  /* receivers (stations), src/seismogram.f90:11-492 */
  int32_t nrec;
  const double *rec_xyz;       /* per receiver x y z; nearest node as Find_Coordinates */
  int32_t fd_operator;         /* WQL3D_FD_*; upwind blocks run the per-point stage kernel and
                                  are not split into s-slabs */
} wql3d_block_desc;

/* Whole-run description (the &problem_list subset the hot path needs). */
typedef struct wql3d_domain_desc {
  int32_t abi_version;         /* WQL3D_ABI_VERSION */
  int32_t nblocks;             /* 1 or 2 (two blocks share a q-direction interface) */
  int32_t precision;           /* WQL3D_FP64 or WQL3D_FP32_COMPENSATED */
  int32_t response;            /* WQL3D_ELASTIC / Q4 / Q8 / FQ8 */
  int32_t coarse_grain;        /* fQ8: 1 when coarse_grain == 2 */
  double Qs0, Qp0;             /* Q4/Q8 scalars when no per-point arrays are given */
  double tau[8];               /* relaxation times */
  double weight[8];            /* Q4/Q8 weights */
  double strength_s[8];        /* fQ8 S strengths */
  double strength_p[8];        /* fQ8 P strengths */
  int32_t coupling;            /* WQL3D_IFACE_* (two blocks) */
  int32_t fault_problem;       /* WQL3D_FAULT_* */
  int32_t serial_shared;       /* 1: both sides' interface solves add to the slip rate (twice per
                                  stage), as in the reference's one-process two-block run;
                                  0: once per stage, as in its one-rank-per-block run */
  double fs, fd, Dc;           /* slip-weakening parameters */
  const double *iface_tau0;    /* optional (3, ns, nr): initial tractions n, m, l on the interface */
  const double *iface_fs;      /* optional (ns, nr) static friction map */
  double fault_stress[6];      /* WQL3D_FAULT_TPV28 background stress (sxx, syy, szz, sxy, sxz, syz);
                                  all zero: (-60, 0, 60, 0, 29.38, 0) of src/initial_stress_condition.f90:78-84 */
  int32_t max_samples;         /* receiver samples kept on the device */
  /* manufactured solution (src/mms.f90:136-235): when mms != 0 every point's
     rates get the forcing u*_t - L(u*) and the face SATs the exact boundary
     data u - u* (src/BoundaryConditions.f90:84-88); such a domain runs the
     generic per-point kernel */
  int32_t mms;
  double mms_nt, mms_nx, mms_ny, mms_nz;
  /* one block per process (the reference's one-rank-per-block run): with
     nblocks = 1, remote_side = 1 makes this block side 1 of a q-interface
     (its q-max face), 2 side 2 (its q-min face); the other side's face trace
     arrives through the interface buffers every stage */
  int32_t remote_side;
  /* one s-slab of a block per process (the reference's spatial decomposition
     with ghost-layer exchange, src/mpi3dcomm.f90:459-528, src/fields.f90:306-321):
     with nblocks = 1 and slab_ns_global > 0, block 0 holds the global s-planes
     slab_z0 + 1 .. slab_z0 + ns of a block of slab_ns_global planes (aqrs / bqrs
     are the whole block's).  Its s faces inside the block are open: no boundary
     condition or PML there, the central SBP row up to the face, and 3 ghost
     planes per open face that wql3d_unpack_halo fills with the neighbour's
     planes.  Curvilinear slabs pass in slab_ghost_coords the coordinates of the
     3 planes below and the 3 above the slab, (3, 6, nr, nq) with q fastest
     (the rows of a side that is a face of the whole block are ignored). */
  int32_t slab_z0;
  int32_t slab_ns_global;
  const double *slab_ghost_coords;
  wql3d_block_desc block[2];
} wql3d_domain_desc;

/* lifecycle (replaces init_domain's device side and enter_domain_device_data,
   src/domain.f90:30-330, src/device_data_openacc.f90:37-87) */
int wql3d_domain_create(const wql3d_domain_desc *desc, wql3d_domain **out);
int wql3d_domain_destroy(wql3d_domain *d);

/* explicit residency (src/device_data_openacc.f90): host <-> device copies */
int wql3d_set_fields(wql3d_domain *d, int block, const double *F, int32_t host_nb);
int wql3d_get_fields(wql3d_domain *d, int block, double *F, int32_t host_nb);
int wql3d_set_rates(wql3d_domain *d, int block, const double *DF, int32_t host_nb);
int wql3d_get_rates(wql3d_domain *d, int block, double *DF, int32_t host_nb);
int wql3d_get_memory_variables(wql3d_domain *d, int block, double *eta);   /* 6 x nmech x n, host_nb 0 */
int wql3d_get_metrics(wql3d_domain *d, int block, double *metrics);       /* 10 x n: metricx, metricy, metricz, J */
int wql3d_get_interface(wql3d_domain *d, double *out);                    /* per point S(4) W Svel trup */
/* one fault output (WQL3D_FO_*) in the layout the reference writes its
   fault files in; replaces write_fault_output / write_hat_output
   (src/domain.f90:782-845).  The face traces (Uface, Vface) are the fields
   at block 1's q-max and block 2's q-min faces (wql3d_get_fields). */
int wql3d_get_fault_output(wql3d_domain *d, int kind, double *out);
/* components c0 .. c0 + ncomp - 1 (0-based; 0..2 velocities, 3..8 stresses)
   of block `block`'s fields on the plane of 1-based index `index` normal to
   axis (1: q, 2: r, 3: s), gathered on the device: out holds n1 x n2 x ncomp
   doubles, the first in-plane index (q, or r for axis 1) fastest.  Replaces
   extract_local_plane (src/plane_output.f90:594-653, the plane writer's
   velocities) and the F(:, location, :, 1:9) sections of write_slice
   (src/slice_output.f90:79-94); the file formats are the host's. */
int wql3d_get_plane(wql3d_domain *d, int block, int axis, int index, int c0, int ncomp, double *out);

/* time integration: one RK stage (time_step.f90:109-147 loop body),
   one time step (time_step_RK) and a graph-captured run of many steps.
   t is the domain time held on the device; wql3d_set_time sets it. */
int wql3d_set_time(wql3d_domain *d, double t);
int wql3d_get_time(wql3d_domain *d, double *t);
int wql3d_stage(wql3d_domain *d, int stage, double dt);
int wql3d_time_step(wql3d_domain *d, double dt, int n, int w_stride);
int wql3d_run(wql3d_domain *d, double dt, int n_first, int nsteps, int w_stride);

/* stage-by-stage driving (domains with a remote interface side, or any
   domain): wql3d_begin_step sets the step counter n and takes the stage-1
   receiver sample (time_step.f90:137); wql3d_stage then runs the stages, the
   fifth advancing the domain time. */
int wql3d_begin_step(wql3d_domain *d, int n, int w_stride);

/* remote interface side (remote_side != 0; src/domain.f90:696-754,
   exchange_fields_interface / exchange_materials_interface): device buffers
   of this block's face trace (send) and the other side's (recv), each
   9 x ns x nr components of elem_bytes (field precision), y fastest;
   wql3d_pack_interface fills send from the current fields on the domain
   stream; the caller moves send to the peer's recv before each wql3d_stage.
   The face material (lambda, mu, rho; 3 x ns x nr doubles) is exchanged once:
   wql3d_get_interface_material gives this side's, wql3d_set_interface_remote_material
   takes the peer's.  wql3d_time_step / wql3d_run are refused (WQL3D_ESTATE). */
int wql3d_interface_buffers(wql3d_domain *d, void **send, void **recv, int64_t *count, int32_t *elem_bytes);
int wql3d_pack_interface(wql3d_domain *d);
int wql3d_get_interface_material(wql3d_domain *d, double *M);
int wql3d_set_interface_remote_material(wql3d_domain *d, const double *M);

/* ghost-plane exchange of an s-slab domain (slab_ns_global > 0;
   src/mpi3dcomm.f90:459-528): device buffers of 2 faces x count elements of
   elem_bytes (field precision), the lower face first, each face
   ncomp x 3 planes x nr x nq with q fastest (ncomp 9 for WQL3D_HALO_FIELDS,
   10 for WQL3D_HALO_METRIC).  wql3d_pack_halo fills send with the 3 planes
   next to each open face; the caller moves send's lower face to the lower
   neighbour's recv upper face and send's upper face to the upper neighbour's
   recv lower face; wql3d_unpack_halo writes recv into the ghost planes.  The
   metric (metricx, metricy, metricz, J) is exchanged once after
   wql3d_domain_create; the fields before every wql3d_stage (after
   wql3d_begin_step).  wql3d_time_step / wql3d_run are refused (WQL3D_ESTATE). */
#define WQL3D_HALO_FIELDS 0
#define WQL3D_HALO_METRIC 1
int wql3d_halo_buffers(wql3d_domain *d, int kind, void **send, void **recv, int64_t *count, int32_t *elem_bytes);
int wql3d_pack_halo(wql3d_domain *d, int kind);
int wql3d_unpack_halo(wql3d_domain *d, int kind);

/* split stage operations (bring-up path, same arithmetic as wql3d_stage) */
int wql3d_scale_rates(wql3d_domain *d, double A);                         /* domain.f90:922-949 */
int wql3d_set_rates_rhs(wql3d_domain *d);                                 /* domain.f90:951-979 */
int wql3d_enforce_bound_iface_conditions(wql3d_domain *d, int stage);     /* domain.f90:615-644 */
int wql3d_update_fields(wql3d_domain *d, double dt);                      /* domain.f90:982-1017 */
/* RHS backend seam: computes the traditional-6 RHS of every block into DF
   and reports handled = 1 (traditional_cartesian_rhs_*.f90) */
int wql3d_try_traditional_rhs(wql3d_domain *d, int *handled);

/* rk_vector backend on raw device arrays (rk_vector_openacc.f90:22-75) */
int wql3d_scale_rate_array(double *rate, int64_t n, double coefficient, void *stream);
/* try_traditional_cartesian_rhs seam of the reference's OpenACC build
   (src/traditional_cartesian_rhs_openacc.f90): adds the strict-interior rates
   of a Cartesian elastic traditional-6 block to `rate`, on the caller's device
   arrays field / rate (n1, n2, n3, 9), metricx / metricy / metricz
   (n1, n2, n3, nm) and material (n1, n2, n3, nmat), Fortran order, for the
   1-based box xlo..xhi x ylo..yhi x zlo..zhi of those arrays (3 points inside
   each side), spacings hq, hr, hs, on `stream`.  Products and sums in the
   reference's order without fused multiply-add. */
int wql3d_traditional_cartesian_rhs(const double *field, double *rate, const double *metricx, const double *metricy,
                                    const double *metricz, const double *material, int32_t n1, int32_t n2, int32_t n3,
                                    int32_t nm, int32_t nmat, int32_t xlo, int32_t xhi, int32_t ylo, int32_t yhi,
                                    int32_t zlo, int32_t zhi, double hq, double hr, double hs, void *stream);
int wql3d_update_state_array(double *state, const double *rate, int64_t n, double increment, void *stream);

/* receivers: samples taken at stage 1 before the update (time_step.f90:137),
   out[(sample*nrec + r)*4 + {t, vx, vy, vz}] */
int wql3d_get_seismograms(wql3d_domain *d, int block, double *out, int32_t *nsamples);
/* start the station sample ring again at sample 0 (a new run of the same domain) */
int wql3d_reset_samples(wql3d_domain *d);
/* run status: waits for the domain's queued work and returns WQL3D_ENONFINITE
   when a station sample of any step so far held a non-finite value (the
   reference stops such a run, src/seismogram.f90:516-524, RUN-STATION-001),
   and WQL3D_ECUDA when a bounded device wait of a stage kernel gave up (the
   fields are then void); bad_step (optional) receives the first non-finite
   step, 0 if none */
int wql3d_check_status(wql3d_domain *d, int32_t *bad_step);
int wql3d_receiver_index(wql3d_domain *d, int block, int32_t *idx);

/* final diagnostics (close_domain): max|F| over all blocks, max|eta|,
   per-block maxima; returns WQL3D_ENONFINITE for non-finite state */
int wql3d_final_state(wql3d_domain *d, double *max_field, double *max_memory, double *block_max);

int wql3d_synchronize(wql3d_domain *d);
int wql3d_get_stream(wql3d_domain *d, void **stream);                    /* the domain's cudaStream_t */
int wql3d_device_bytes(wql3d_domain *d, int64_t *bytes);
int wql3d_kernel_launches(wql3d_domain *d, int64_t *launches);
const char *wql3d_last_error(void);

/* Curvilinear block mesh by 3-D transfinite interpolation on the device
   (Gen3_Curve_Mesh of Curve_Grid_3D3, src/grid.f90:2292-2418, :473-1909):
   faces holds the six boundary surfaces, x / y / z each, in the order left,
   right (q = 0 / 1; ns x nr, r fastest), top, bottom (r = 0 / 1; ns x nq),
   front, back (s = 0 / 1; nr x nq); coords receives 3 x ns x nr x nq with q
   fastest (the wql3d_block_desc.coords layout with host_nb 0).  A set-up
   call: it allocates and frees its device buffers. */
int wql3d_tfi_grid(const double *faces, int32_t nq, int32_t nr, int32_t ns, double *coords);

/* Parameter updates between runs (the inversion loop of an adjoint driver):
   material lambda, mu, rho of one block (3 components, host_nb 0) and the
   moment tensors of its sources (nsrc x 6: mxx myy mzz mxy mxz myz). */
int wql3d_set_material(wql3d_domain *d, int block, const double *M);
int wql3d_set_moment(wql3d_domain *d, int block, const double *m6);

/* Device-resident field checkpoints (FP64): the current field buffer of a
   block copied to / from a caller device array of wql3d_field_volume
   elements (the library's padded layout) on the domain stream. */
int wql3d_field_volume(wql3d_domain *d, int block, int64_t *elements);
int wql3d_store_fields(wql3d_domain *d, int block, double *dev_dst);
int wql3d_load_fields(wql3d_domain *d, int block, const double *dev_src);

/* Discrete adjoint of the elastic RK step.  No counterpart in the reference,
   which has no adjoint: it serves waveform-misfit gradients with respect to
   lambda, mu, rho and the sources' moment tensors.  It is the transpose of the
   stage operator with every point in the conservative near-boundary form of
   src/JU_xJU_yJU_z6.f90:12-809 (the curvilinear stage itself; rounding-level
   different from the Cartesian interior form), the face SATs of
   src/RHS_Interior.f90:1584-1768 and the sources of src/moment_tensor.f90:875-1125,
   for one FP64 elastic traditional-6 block without PML (WQL3D_EINVAL otherwise).
   Usage: enable once; reset; then for n = N..1 with the domain's fields set
   to F_n (the state at the start of step n) and its time to t_n:
   wql3d_adjoint_step (adjoint of step n: recomputes the five stage inputs
   and reverses the stages, accumulating the gradients), then
   wql3d_adjoint_add_receivers with the misfit derivative with respect to
   sample n (the stage-1 station velocities v(t_n), nrec x 3).  The field
   adjoint after n = 1 is the misfit derivative with respect to F_1. */
int wql3d_adjoint_enable(wql3d_domain *d);
int wql3d_adjoint_reset(wql3d_domain *d);
int wql3d_adjoint_step(wql3d_domain *d, int n, double dt);
int wql3d_adjoint_add_receivers(wql3d_domain *d, int block, const double *res);
/* The same reversal without recomputing the stage inputs: wql3d_record_step
   runs time step n like wql3d_time_step (one-block FP64 domain) and records
   into dev_out (WQL3D_RECORD_FIELDS x wql3d_field_volume doubles on the
   device) its five stage inputs F^(0..4) and, for a curvilinear block, the
   derivative terms of each stage input that the material gradient needs (the
   stage kernel writes them as it computes them: strain rates and stress-flux
   sums, 9 components); wql3d_adjoint_step_recorded reverses step n from such
   a record (t_n: the time at the start of step n) without re-deriving them.
   A driver records a checkpoint segment once and reverses it from the
   records. */
#define WQL3D_RECORD_FIELDS 10
int wql3d_record_step(wql3d_domain *d, double dt, int n, int w_stride, double *dev_out);
int wql3d_adjoint_step_recorded(wql3d_domain *d, int n, double dt, double t_n, const double *dev_in);
/* L^T R and (dL/d(lambda, mu, rho) F)^T R at the current fields, host arrays
   (R, Fbar: 9 x n; g: 3 x n; host_nb 0) */
int wql3d_adjoint_rhs(wql3d_domain *d, int block, const double *R, double *Fbar, double *g);
int wql3d_get_adjoint_fields(wql3d_domain *d, int block, double *Fbar);
/* accumulated gradients: g_material 3 x n (lambda, mu, rho), g_moment nsrc x 6 */
int wql3d_get_adjoint_gradient(wql3d_domain *d, int block, double *g_material, double *g_moment);

/* Batched independent shots.  No counterpart in the reference, which runs
   one problem per process: the batched-shot configuration advances many
   one-block Cartesian traditional-6 domains (same precision and time step,
   no PML; responses may differ) with one launch per kernel kind and RK stage
   for all of them, captured two steps at a time in one CUDA graph.  Work
   lists assign every CTA to one shot (interior tiles, 128-point chunks of the
   near-boundary shell).  The first run tunes the interior tiles' z-chunk
   length over its first steps (each candidate times one step; the arithmetic
   of a point does not depend on it) and keeps the fastest.  The batch orders
   its work after the shots' own queued work and theirs after the batch; the
   shots' domains stay usable for set/get calls.  Domains must outlive the
   batch. */
typedef struct wql3d_batch wql3d_batch;
int wql3d_batch_create(wql3d_domain *const *domains, int32_t n, wql3d_batch **out);
int wql3d_batch_run(wql3d_batch *bt, double dt, int32_t nsteps, int32_t w_stride);
/* chosen z-chunk and the tuning record: ntried candidates zs[i] with their step times ms[i] */
int wql3d_batch_tuning(wql3d_batch *bt, int32_t *zchunk, int32_t *ntried, int32_t *zs, float *ms);
int wql3d_batch_launches(wql3d_batch *bt, int64_t *launches);
int wql3d_batch_synchronize(wql3d_batch *bt);
int wql3d_batch_destroy(wql3d_batch *bt);

/* Allocation-free max|v| reduction over a device array.
   No counterpart in the reference: it serves callers that cannot allocate GPU
   memory when they need the diagnostic (for example a Fortran driver whose
   device data is owned by fixed OpenACC data regions and audited for zero
   allocations during time stepping).  The scratch is a static device array
   inside libwql3d.so (1 MiB on every GPU that loads the library, held until
   exit); the call allocates nothing.  array: device array of n doubles;
   result and nonfinite: device-accessible outputs written on `stream`
   (max |array[i]| and 1 if any element is NaN/Inf).  n may not exceed
   WQL3D_NOALLOC_MAX_ELEMENTS (WQL3D_EINVAL otherwise).  The first call on a
   device looks up the scratch address for that device and loads the
   library's kernels onto it (with lazy module loading this is when the
   driver places the scratch and the kernel code on the device), so make it
   before any stream capture and before the window in which the caller must
   not allocate; later calls allocate nothing.  The address is cached per
   device: after cudaDeviceReset the entry point must not be called again in
   that process.  Calls whose kernels overlap on the GPU share the scratch
   and race; calls ordered on one stream are safe. */
#define WQL3D_NOALLOC_MAX_ELEMENTS (65536LL * 8192LL)
int wql3d_max_abs_noalloc(const double *array, int64_t n, double *result, int32_t *nonfinite, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* WQL3D_H */
