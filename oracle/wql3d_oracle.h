/*
 * CPU oracle for the WaveQLab3D per-step volume update (test infrastructure).
 *
 * This is a plain-C restatement of the reference Fortran solver's hot path,
 * used only by the tests, by __graft_entry__.smoke() and by bench.py's CPU
 * baseline leg, always as the checker and never as the product.  Every
 * routine cites the reference source (paths relative to the reference
 * project root) that it follows.
 *
 * Array convention: one block of nq x nr x ns points, Fortran order (q/x
 * fastest), 1-based indices with nb = 3 ghost layers, exactly like the
 * reference's allocate_array_body (src/mpi3dcomm.f90:631-735).
 */
#ifndef WQL3D_ORACLE_H
#define WQL3D_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_ELASTIC = 0, ORC_Q4 = 1, ORC_Q8 = 2, ORC_FQ8 = 3 };

/* source time functions, src/moment_tensor.f90:813-873 (+ ricker, an addition) */
enum {
  ORC_STF_GAUSSIAN = 0, ORC_STF_LOH_DISC = 1, ORC_STF_BRUNE = 2, ORC_STF_COSBELL = 3,
  ORC_STF_COSINE = 4, ORC_STF_LOH_MOMENT = 5, ORC_STF_SINE_MOMENT = 6, ORC_STF_RICKER = 7
};

/* interface coupling laws, src/Interface_Condition.f90 */
enum { ORC_FD_TRADITIONAL6 = 0, ORC_FD_UPWIND4 = 1, ORC_FD_UPWIND6 = 2, ORC_FD_UPWIND_DRP6 = 3 };
enum { ORC_IFACE_LOCKED = 0, ORC_IFACE_SLIP_WEAKENING = 1, ORC_IFACE_LINEAR = 2, ORC_IFACE_RATE_STATE = 3 };
enum { ORC_FAULT_MAPS = 0, ORC_FAULT_TPV5 = 1, ORC_FAULT_TPV101 = 2, ORC_FAULT_TPV102 = 3, ORC_FAULT_TPV28 = 4 };
/* fault outputs, src/domain.f90:782-845 and src/fault_output.f90:73-122; layout [comp][ns][nr] */
enum { ORC_FO_S = 0, ORC_FO_SVEL = 1, ORC_FO_UHAT = 2, ORC_FO_VHAT = 3, ORC_FO_STATE = 4, ORC_FO_TRUP = 5 };

typedef struct {
  int nq, nr, ns;
  int mesh;        /* 0: 'cartesian' interior form, 1: 'curvilinear' */
  int f32lit;      /* 1: closure literal 0.013435342414630 in single precision */
  int bc[6];       /* type_of_bc on Lx,Rx,Ly,Ry,Lz,Rz; -1: none, 0: interface */
  int pml[6];      /* PML slab flags, faces 1..6 */
  int npml;
  int response;    /* ORC_ELASTIC / ORC_Q4 / ORC_Q8 / ORC_FQ8 */
  int coarse;      /* fQ8 coarse_grain == 2 */
  double aqrs[3], bqrs[3];
  double rho_s_p[3];
  const double *coords;   /* optional: 3*nq*nr*ns coordinates (x fastest, component slowest) */
  const double *material; /* optional: 3*nq*nr*ns (lambda, mu, rho) */
  const double *qsinv;    /* optional: nq*nr*ns Qs^-1 (Q4/Q8) */
  const double *qpinv;    /* optional: nq*nr*ns Qp^-1 (Q4/Q8) */
  double tau[8], weight[8], sstr[8], pstr[8];
  double tau0;
  int nsrc, src_order, src_alpha;
  const int *src_type;     /* per source: ORC_STF_* */
  const double *src_par;   /* per source 11 values: duration t_init mxx myy mzz mxy mxz myz x y z */
  int nrec;
  const double *rec_xyz;   /* per receiver 3 values */
  /* manufactured solution (src/mms.f90:136-235): forcing added to the rates and
     exact boundary data in the face SATs when mms != 0 */
  int mms;
  double mms_nt, mms_nx, mms_ny, mms_nz;
  /* derivative operator (fd_type / order of &problem_list): ORC_FD_TRADITIONAL6,
     or an upwind pair, velocities by the forward and stresses by the backward
     operator: ORC_FD_UPWIND4 (src/JU_xJU_yJU_z6.f90:1439-2033, :17865-18400),
     ORC_FD_UPWIND6 (:2665-3688, :18958-19510), ORC_FD_UPWIND_DRP6 (:10556-12058
     and JJU_x6_interior_upwind_drp) */
  int fd;
} orc_desc;

typedef struct {
  int coupling;            /* ORC_IFACE_* */
  int double_ds;           /* 1: one-process two-block run (src/domain.f90:615-644): Interface_RHS runs
                              once per block side on the shared iface, so DS and DW grow twice per stage */
  int problem;             /* ORC_FAULT_MAPS: prestress/static friction from the maps below;
                              ORC_FAULT_TPV5: src/Interface_Condition.f90:1283-1299, 1822-1830;
                              ORC_FAULT_TPV28: :1459-1474, 2049-2076 */
  /* slip-weakening / linear friction parameters (uniform over the fault) */
  double fs, fd, Dc, alpha_lin;
  const double *tau0_n;    /* optional per-face-point initial normal traction (nr*ns) */
  const double *tau0_l;    /* optional initial shear traction along l (nr*ns) */
  const double *tau0_m;    /* optional initial shear traction along m (nr*ns) */
  const double *fs_map;    /* optional per-point static friction (nr*ns) */
  /* ORC_FAULT_TPV28 background stress (sxx, syy, szz, sxy, sxz, syz); all zero:
     the tensor of src/initial_stress_condition.f90:78-84 */
  double s0[6];
} orc_iface_desc;

void *orc_create(int nblocks, const orc_desc *blocks, const orc_iface_desc *iface);
void orc_destroy(void *d);
double orc_time(void *d);
void orc_set_time(void *d, double t);
/* advance nsteps of time_step_RK; seismograms sampled at stage 1 of every w_stride-th step:
   seis[(sample*nrec + r)*4 + {t,vx,vy,vz}] for block `b` receivers (b = 0 or 1) */
int orc_run(void *d, double dt, int nsteps, int w_stride, double *seis0, double *seis1);
/* single RK stage (stage in 1..5) at stage time t; used by per-stage tests */
void orc_stage(void *d, int stage, double dt);
void orc_get_fields(void *d, int b, double *out);       /* 9*nq*nr*ns */
void orc_set_fields(void *d, int b, const double *in);
void orc_get_rates(void *d, int b, double *out);        /* 9*nq*nr*ns */
void orc_set_rates(void *d, int b, const double *in);
void orc_get_metrics(void *d, int b, double *out);      /* 10*nq*nr*ns: metricx(1:3) metricy(1:3) metricz(1:3) J */
void orc_get_material(void *d, int b, double *out);     /* 3*nq*nr*ns */
int orc_get_eta(void *d, int b, double *out);           /* 6*nmech*nq*nr*ns, returns nmech */
void orc_set_eta(void *d, int b, const double *in);
void orc_get_pml(void *d, int b, int face, double *out);/* 9*npts of slab */
void orc_get_normals(void *d, int b, int face, double *out); /* 9*face points: n_l(3) n_m(3) n_n(3) */
void orc_get_iface(void *d, double *out);               /* per point: S(4) W(1) Svel(1) trup(1) */
/* one fault output (ORC_FO_*): S 4, Svel 3, Uhat 6, Vhat 6, state 1, trup 1 components;
   Svel/Uhat/Vhat are the values recorded at stage 1 of the last step */
int orc_get_fault(void *d, int kind, double *out);
void orc_receiver_index(void *d, int b, int *idx);      /* 3 per receiver */
void orc_final_state(void *d, double *maxF, double *maxEta, double *maxB);
/* manufactured solution at time t on block b's grid: 9*nq*nr*ns (src/mms.f90:136-148) */
void orc_mms_exact(void *d, int b, double t, double *out);

/* coefficient builders, src/anelastic_q4_model.f90:97-111, src/anelastic_q8_model.f90:100-116 */
/* row of an upwind operator (ORC_FD_UPWIND*; plus: D+ or D-) at 1-based i of
   n points, up to 13 taps; returns the tap count (0 for traditional-6) */
int orc_upwind_row(int fd, int plus, int i, int n, int *idx, double *c);
void orc_q4_coefficients(double fmin, double fmax, double *tau, double *weight);
void orc_q8_coefficients(double fmin, double fmax, double *tau, double *weight);
/* modulus correction, src/material.f90:156-298 (Q4), :330-485 (Q8) */
void orc_modulus_correction(int nmech, const double *tau, const double *weight, double fref,
                            long n, double *lam, double *mu, const double *rho,
                            const double *qsinv, const double *qpinv);

#ifdef __cplusplus
}
#endif
#endif
