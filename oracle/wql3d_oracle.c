/*
 * CPU oracle for the WaveQLab3D per-step volume update.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain C, the reference
 * Fortran solver's hot path so that the CUDA product can be checked against
 * it.  It is imported only by tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py.  Nothing in the product
 * links it.
 *
 * Parity is pinned by the reference's own published 16-digit known answer
 * (inputfile/test_elastic_traditional_o6.in ->
 * "Elastic final state: max|field|=1.6623128367649574E+02",
 * PHASE5_TRADITIONAL_CARTESIAN_RHS.md:35) and by the rupture truth files
 * test_problems/truth/{1,2} (see tests/golden/).
 *
 * Every routine names the reference file:line it follows.  Floating-point
 * expressions keep the reference's evaluation order (Fortran evaluates
 * left to right within one precedence level), and the file is compiled with
 * -ffp-contract=off so no fused multiply-add changes the rounding.
 */
#include "wql3d_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NB 3
#define PI_WP 3.141592653589793

/* ------------------------------------------------------------------------ */
/* 6th-order SBP first-derivative operator (traditional-6).                  */
/* Boundary rows 1..6 in the order their terms are written in                */
/* src/JU_xJU_yJU_z6.f90:74-161 (left closure) and src/metrics.f90:29-86.    */
/* Right rows are the negated mirror, src/JU_xJU_yJU_z6.f90:170-290.          */
/* The row-4 coefficient 0.013435342414630 carries no _wp kind suffix in the */
/* reference, so without -fdefault-real-8 it is a single-precision literal.  */
/* ------------------------------------------------------------------------ */
typedef struct { int n; int idx[8]; double c[8]; } sbp_row;

static sbp_row g_left[6];
static int g_f32lit_cached = -1;

static void sbp_init(int f32lit) {
  if (g_f32lit_cached == f32lit) return;
  const double c4_7 = f32lit ? (double)0.013435342414630f : 0.013435342414630;
  sbp_row r1 = {6, {6, 5, 4, 3, 2, 1}, {0.036577936277544, 0.104488069284042, -0.450398306578272,
                                        -0.141512858744873, 2.033378678700676, -1.582533518939116}};
  sbp_row r2 = {5, {6, 5, 4, 3, 1}, {-0.014903449191300, -0.069112065532624, 0.258816087376832,
                                     0.287258622978251, -0.462059195631158}};
  sbp_row r3 = {5, {6, 5, 4, 2, 1}, {-0.018129342917256, -0.022902190275815, 0.606235523609147,
                                     -0.636451095137907, 0.071247104721830}};
  sbp_row r4 = {6, {7, 6, 5, 3, 2, 1}, {c4_7, -0.051642265516119, 0.520262285050482,
                                        -0.306681191361148, -0.290087484386815, 0.114713313798970}};
  sbp_row r5 = {7, {8, 7, 6, 4, 3, 2, 1}, {0.018281071473911, -0.164529643265203, 0.769199413962647,
                                           -0.707905442575989, 0.015764336127392, 0.105400944933782,
                                           -0.036210680656541}};
  sbp_row r6 = {8, {9, 8, 7, 5, 4, 3, 2, 1}, {0.016437980868017, -0.147941827812150, 0.739709139060752,
                                              -0.691649024426814, 0.063183694641876, 0.011220896474665,
                                              0.020437334208704, -0.011398193015050}};
  g_left[0] = r1; g_left[1] = r2; g_left[2] = r3; g_left[3] = r4; g_left[4] = r5; g_left[5] = r6;
  g_f32lit_cached = f32lit;
}

/* The stencil row used at 1-based position i of an axis with n points:
   absolute 1-based indices and signed coefficients, in summation order. */
static void sbp_stencil(int i, int n, int *cnt, int *idx, double *c) {
  static const double cc[6] = {-1.0 / 60.0, 0.15, -0.75, 0.75, -0.15, 1.0 / 60.0};
  static const int off[6] = {-3, -2, -1, 1, 2, 3};
  if (i >= 7 && i <= n - 6) {
    *cnt = 6;
    for (int k = 0; k < 6; ++k) { idx[k] = i + off[k]; c[k] = cc[k]; }
    return;
  }
  if (i >= n - 5) { /* right closure (mirror of left row n+1-i) */
    const sbp_row *r = &g_left[n - i];
    *cnt = r->n;
    for (int k = 0; k < r->n; ++k) { idx[k] = n + 1 - r->idx[k]; c[k] = -r->c[k]; }
    return;
  }
  const sbp_row *r = &g_left[i - 1];
  *cnt = r->n;
  for (int k = 0; k < r->n; ++k) { idx[k] = r->idx[k]; c[k] = r->c[k]; }
}

/* ------------------------------------------------------------------------ */
/* Upwind SBP operator pairs: velocities take the forward operator D+,       */
/* stresses the backward operator D-.  Per operator: the width of the        */
/* closure (rows 1..w at each end; the strict interior starts at w + 1), the */
/* interior stencils (first offsets and coefficients, as the near-boundary   */
/* routine writes them and as the interior routine does), and the left       */
/* closure rows of both operators in the order the reference writes their    */
/* terms.  The right closure of each operator is the negated mirror of the   */
/* other operator's left rows, terms in the same order.                      */
/*   upwind-4:     src/JU_xJU_yJU_z6.f90:1439-2033, :17865-18400             */
/*   upwind-6:     src/JU_xJU_yJU_z6.f90:2665-3688, :18958-19510             */
/*   upwind-DRP-6: src/JU_xJU_yJU_z6.f90:10556-12058, and its interior       */
/*                 routine JJU_x6_interior_upwind_drp                         */
/* ------------------------------------------------------------------------ */
#define UP_MAXT 13
typedef struct { int n; int idx[UP_MAXT]; double c[UP_MAXT]; } up_row;
typedef struct {
  int width;                        /* closure rows per end */
  int taps;                         /* interior taps */
  int of, ob;                       /* first interior offset of D+ / D- */
  double nbf[10], nbb[10];          /* interior rows of the near-boundary routine */
  double inf_[10], inb[10];         /* coefficients of the strict-interior routine */
  const up_row *plus, *minus;       /* left closure rows 1..width */
} upwind_op;

static const up_row g_up4_plus[4] = {
    {4, {4, 3, 2, 1}, {0.030612244897959, -0.591836734693878, 2.091836734693878, -1.530612244897959}},
    {5, {5, 4, 3, 2, 1}, {0.065573770491803, -0.234972677595628, 0.811475409836066, -0.180327868852459,
                          -0.461748633879781}},
    {6, {6, 5, 4, 3, 2, 1}, {0.097560975609756, -0.585365853658537, 1.581300813008130, -0.707317073170732,
                             -0.475609756097561, 0.089430894308943}},
    {7, {7, 6, 5, 4, 3, 2, 1}, {0.080536912751678, -0.483221476510067, 1.449664429530201, -0.785234899328859,
                                -0.218120805369128, -0.073825503355705, 0.030201342281879}}};
static const up_row g_up4_minus[4] = {
    {4, {4, 3, 2, 1}, {-0.091836734693878, -0.224489795918367, 1.724489795918367, -1.408163265306122}},
    {4, {4, 3, 2, 1}, {0.060109289617486, 0.319672131147541, 0.180327868852459, -0.560109289617486}},
    {4, {4, 3, 2, 1}, {0.264227642276423, 0.707317073170732, -1.207317073170732, 0.235772357723577}},
    {5, {5, 4, 3, 2, 1}, {0.241610738255034, 0.785234899328859, -1.305369127516778, 0.288590604026846,
                          -0.010067114093960}}};

static const up_row g_up6_plus[6] = {
    {6, {6, 5, 4, 3, 2, 1}, {0.054021710000147, 0.023993033880123, -0.302855902188632, -0.275607596716317,
                             2.093702214477299, -1.593253459452621}},
    {6, {6, 5, 4, 3, 2, 1}, {-0.039560344515975, 0.030739159126096, 0.105980141988699, 0.393228064437077,
                             -0.029551468764759, -0.460835552271137}},
    {7, {7, 6, 5, 4, 3, 2, 1}, {-0.026915887850467, 0.197069524204597, -0.589452745232692, 1.258766829227482,
                                -0.306540940575249, -0.629259919521358, 0.096333139747688}},
    {8, {8, 7, 6, 5, 4, 3, 2, 1}, {-0.013345690454124, 0.106765523632994, -0.330443502642251, 0.946962507015985,
                                   -0.318292975073623, -0.243684445410829, -0.240558007429252, 0.092596590361100}},
    {9, {9, 8, 7, 6, 5, 4, 3, 2, 1}, {-0.018365004463716, 0.146920035709731, -0.550950133911491, 1.406282074938901,
                                      -0.593528379527062, -0.450132219590077, 0.041897570295664, 0.033485250803205,
                                      -0.015609194255155}},
    {10, {10, 9, 8, 7, 6, 5, 4, 3, 2, 1}, {-0.016424481602299, 0.131395852818395, -0.492734448068983,
                                           1.313958528183954, -0.572337434946968, -0.357460227911152,
                                           -0.025427590054054, -0.005338567444210, 0.040531470682718,
                                           -0.016163101657400}}};
static const up_row g_up6_minus[6] = {
    {6, {6, 5, 4, 3, 2, 1}, {0.052048915548040, 0.044953974933765, -0.366971721882124, -0.189297839436616,
                             2.039450367044345, -1.580183696207410}},
    {6, {6, 5, 4, 3, 2, 1}, {-0.029492540133095, -0.021790841692085, 0.215422101432619, 0.279404147185598,
                             0.029551468764759, -0.473094335557797}},
    {6, {6, 5, 4, 3, 2, 1}, {0.008748664712219, -0.061405392278187, 0.491468255323896, 0.306540940575249,
                             -0.885608401570530, 0.140255933237354}},
    {6, {6, 5, 4, 3, 2, 1}, {0.020661154127888, 0.327107204245208, 0.318292975073623, -0.624133691970994,
                             -0.118346128899150, 0.076418487423426}},
    {7, {7, 6, 5, 4, 3, 2, 1}, {-0.036730008927433, 0.399693508760138, 0.593528379527062, -1.303115093827634,
                                0.402190050630647, -0.047235828122731, -0.008331008040049}},
    {8, {8, 7, 6, 5, 4, 3, 2, 1}, {-0.032848963204599, 0.394187558455186, 0.572337434946968, -1.257688453771463,
                                   0.406675342006739, -0.120254802392339, 0.054367610816546, -0.016775726857039}}};
static const up_row g_drp6_plus[8] = {
    {8, {8, 7, 6, 5, 4, 3, 2, 1}, {
        -0.033005239880522, -0.025881634391799, 0.263392722344631, -0.030209714180198,
        -0.506938949737935, -0.350517535783371, 2.412053651292632, -1.728893299663438}},
    {8, {8, 7, 6, 5, 4, 3, 2, 1}, {
        0.008828095360976, 0.029911851210588, -0.170162903794152, 0.094426023794218,
        0.250037914252055, 0.250891381680726, -0.020053857114091, -0.443878505390320}},
    {8, {8, 7, 6, 5, 4, 3, 2, 1}, {
        -0.086554962191340, 0.357259827206167, -0.022134128148434, -1.484851853641141,
        2.378309161955782, -0.045718284610534, -1.531087089237169, 0.434777328666669}},
    {9, {9, 8, 7, 6, 5, 4, 3, 2, 1}, {
        -0.002634349609551, 0.079463252429367, -0.299393382304440, 0.407288103594466,
        0.281750824243924, -0.012373610391183, -0.330330927617320, -0.204468804842354,
        0.080698894497091}},
    {10, {10, 9, 8, 7, 6, 5, 4, 3, 2, 1}, {
        -0.011812293127050, 0.027365145744332, -0.517048981121307, 1.165933921548919,
        0.122648484113833, -0.373648890457135, -1.160735576719516, 1.025653483809176,
        -0.176618285456005, -0.101737008335247}},
    {11, {11, 10, 9, 8, 7, 6, 5, 4, 3, 2, 1}, {
        -0.003705846074975, 0.008585210073693, 0.061269988439591, -0.203098167192540,
        0.696367795879953, -0.264391437780108, 0.124789282744944, -0.548404955515763,
        0.002073955135157, 0.176979071835593, -0.050464897545544}},
    {12, {12, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2, 1}, {
        -0.005172307293959, 0.011982511897672, 0.085515480593458, -0.535851035654166,
        1.560836153489656, -0.905179927543220, -0.052231816759526, -0.486889270320233,
        0.517428663501413, -0.137956948397386, -0.108190216650142, 0.055708713136433}},
    {13, {13, 12, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2, 1}, {
        -0.004715630209601, 0.010924543318908, 0.077965086132063, -0.488539289714622,
        1.474420378868455, -0.892828448398233, -0.032767235755012, -0.248685062282352,
        0.170930500243401, -0.110359853738840, 0.038849792028224, 0.017743142086478,
        -0.012937922578870}}};
static const up_row g_drp6_minus[8] = {
    {8, {8, 7, 6, 5, 4, 3, 2, 1}, {
        0.044374156234105, -0.174198378773702, 0.220245640409051, 0.139299657443443,
        -0.495449593250587, -0.370787168310084, 2.304067463556378, -1.667551777308605}},
    {8, {8, 7, 6, 5, 4, 3, 2, 1}, {
        -0.011723708576681, 0.065174528307485, -0.148801997699767, 0.046588172420165,
        0.241839854684496, 0.251551333921227, 0.020053857114091, -0.464682040171017}},
    {8, {8, 7, 6, 5, 4, 3, 2, 1}, {
        -0.156241518792227, 0.505832529848511, -0.010613520806507, -1.646697927315869,
        2.378062811419621, 0.045718284610534, -1.527070237729393, 0.411009578765331}},
    {8, {8, 7, 6, 5, 4, 3, 2, 1}, {
        0.061651661535115, -0.263535772373310, 0.389840903051706, 0.258864496540571,
        0.012373610391183, -0.330365147571788, -0.211400033956727, 0.082570282383251}},
    {9, {9, 8, 7, 6, 5, 4, 3, 2, 1}, {
        0.014765366408812, -0.428167834093026, 1.111936792339292, -0.397762766470929,
        0.373648890457135, -1.263356736209345, 0.924846902011930, -0.357974171524791,
        0.022063557080921}},
    {10, {10, 9, 8, 7, 6, 5, 4, 3, 2, 1}, {
        0.004632307593719, -0.036811404344754, 0.195432746208080, 0.037422964670561,
        0.264391437780108, -0.038478253000180, -0.572948637727217, 0.004325161232786,
        0.202384868750895, -0.060351191163998}},
    {11, {11, 10, 9, 8, 7, 6, 5, 4, 3, 2, 1}, {
        0.006465384117449, -0.051378252453327, 0.137238553533049, 0.035940522255854,
        0.905179927543220, -0.971931417829373, -0.510533260717342, 0.587831838812040,
        -0.097436350250351, -0.049653902328415, 0.008276957317196}},
    {12, {12, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2, 1}, {
        0.005894537762001, -0.046841926748699, 0.125121388228069, 0.105630116695053,
        0.892828448398233, -1.423025682605699, 0.258439188609325, 0.206413079068906,
        -0.142243577826732, 0.021522078805545, -0.013360802114642, 0.009623151728641}}};

/* D+ of the interior routines is -(D-) mirrored: nbb / inb are the reversed,
   negated nbf / inf_ (kept written out as each routine writes them) */
static const upwind_op g_upwind4 = {
    4, 5, -1, -3,
    {-0.250000000000000, -0.833333333333333, 1.500000000000000, -0.500000000000000, 0.083333333333333},
    {-0.083333333333333, 0.500000000000000, -1.500000000000000, 0.833333333333333, 0.250000000000000},
    {-1.0 / 4.0, -5.0 / 6.0, 3.0 / 2.0, -1.0 / 2.0, 1.0 / 12.0},
    {-1.0 / 12.0, 1.0 / 2.0, -3.0 / 2.0, 5.0 / 6.0, 1.0 / 4.0},
    g_up4_plus, g_up4_minus};
static const upwind_op g_upwind6 = {
    6, 7, -2, -4,
    {1.0 / 30.0, -2.0 / 5.0, -7.0 / 12.0, 4.0 / 3.0, -1.0 / 2.0, 2.0 / 15.0, -1.0 / 60.0},
    {1.0 / 60.0, -2.0 / 15.0, 1.0 / 2.0, -4.0 / 3.0, 7.0 / 12.0, 2.0 / 5.0, -1.0 / 30.0},
    {1.0 / 30.0, -0.4, -7.0 / 12.0, 4.0 / 3.0, -0.5, 2.0 / 15.0, -1.0 / 60.0},
    {1.0 / 60.0, -2.0 / 15.0, 0.5, -4.0 / 3.0, 7.0 / 12.0, 0.4, -1.0 / 30.0},
    g_up6_plus, g_up6_minus};
static const upwind_op g_drp6 = {
    8, 10, -4, -5,
    {-0.005952380952381, 0.047301587301587, -0.126349206349206, -0.106666666666667, -0.888888888888889,
     1.488888888888889, -0.493333333333333, 0.078730158730159, 0.011031746031746, -0.004761904761905},
    {0.004761904761905, -0.011031746031746, -0.078730158730159, 0.493333333333333, -1.488888888888889,
     0.888888888888889, 0.106666666666667, 0.126349206349206, -0.047301587301587, 0.005952380952381},
    {-1.0 / 168.0, 149.0 / 3150.0, -199.0 / 1575.0, -8.0 / 75.0, -8.0 / 9.0, 67.0 / 45.0, -37.0 / 75.0,
     124.0 / 1575.0, 139.0 / 12600.0, -1.0 / 210.0},
    {1.0 / 210.0, -139.0 / 12600.0, -124.0 / 1575.0, 37.0 / 75.0, -67.0 / 45.0, 8.0 / 9.0, 8.0 / 75.0,
     199.0 / 1575.0, -149.0 / 3150.0, 1.0 / 168.0},
    g_drp6_plus, g_drp6_minus};

/* the block's upwind operator, NULL for traditional-6 */
static const upwind_op *upwind_of(int fd) {
  if (fd == ORC_FD_UPWIND4) return &g_upwind4;
  if (fd == ORC_FD_UPWIND6) return &g_upwind6;
  if (fd == ORC_FD_UPWIND_DRP6) return &g_drp6;
  return NULL;
}

/* Row of D+ (plus = 1) or D- (plus = 0) at 1-based i of n points, with the
   near-boundary routine's interior coefficients */
static void up_stencil(const upwind_op *op, int plus, int i, int n, int *cnt, int *idx, double *c) {
  const int w = op->width;
  if (i > w && i <= n - w) {
    *cnt = op->taps;
    for (int k = 0; k < op->taps; ++k) {
      idx[k] = i + (plus ? op->of : op->ob) + k;
      c[k] = plus ? op->nbf[k] : op->nbb[k];
    }
    return;
  }
  if (i > n - w) { /* negated mirror of the other operator's left row n+1-i */
    const up_row *r = plus ? &op->minus[n - i] : &op->plus[n - i];
    *cnt = r->n;
    for (int k = 0; k < r->n; ++k) { idx[k] = n + 1 - r->idx[k]; c[k] = -r->c[k]; }
    return;
  }
  const up_row *r = plus ? &op->plus[i - 1] : &op->minus[i - 1];
  *cnt = r->n;
  for (int k = 0; k < r->n; ++k) { idx[k] = r->idx[k]; c[k] = r->c[k]; }
}

/* ------------------------------------------------------------------------ */
/* Block storage                                                             */
/* ------------------------------------------------------------------------ */
typedef struct {
  int x0, x1, y0, y1, z0, z1; /* inclusive 1-based box */
  int active;
} box_t;

typedef struct {
  orc_desc d;
  int nx, ny, nz, NX, NY, NZ;
  long np;                  /* padded point count */
  double hq, hr, hs;
  double *X[3];
  double *mx[3], *my[3], *mz[3], *J;
  double *M[3];
  double *F[9], *DF[9];
  /* PML slabs, faces 1..6 */
  box_t pbox[6];
  double *Q[6][9], *DQ[6][9];
  /* anelastic */
  int nmech;
  double *qs, *qp;
  double *eta[6][8], *deta[6][8];
  /* boundary faces: normals n_l, n_m, n_n (3 comps each), face-local 2-D */
  double *nl[6][3], *nm[6][3], *nn[6][3];
  int fdim[6][2];
  double *work[6][9];       /* SAT forcing u_bc per face */
  /* sources */
  int nsrc;
  int *stype;
  double *spar;
  int *snear;               /* 3 per source */
  double *sphys;            /* 3 per source */
  /* receivers */
  int nrec;
  int *ridx;
  /* interface face buffers (for 2-block runs) */
  double *faceF[2][9];      /* own face (q-min: 0, q-max: 1) copied fields */
  double *faceFopp[2][9];
  double *faceM[2][3];
  double *faceMopp[2][3];
} oblk;

typedef struct {
  orc_iface_desc d;
  int nr, ns;
  double *S[4], *DS[4], *W, *DW, *Svel[3], *trup;
  double *Uhat[6], *Vhat[6];  /* stage-1 fault outputs (fault%Uhat_pluspres, Vhat_pluspres) */
  double *t0n, *t0m, *t0l, *fsm;
} oiface;

typedef struct {
  int nb;
  oblk *B[2];
  oiface *I;
  double t;
} odom;

static inline long ID(const oblk *b, int x, int y, int z) {
  return (long)(x - 1 + NB) + (long)b->NX * ((long)(y - 1 + NB) + (long)b->NY * (long)(z - 1 + NB));
}
static inline long FID(const oblk *b, int face, int a, int c) {
  /* face-local index: faces 1,2 -> (y,z); 3,4 -> (x,z); 5,6 -> (x,y), 1-based */
  (void)b;
  return (long)(a - 1) + (long)b->fdim[face][0] * (long)(c - 1);
}
static inline long PID(const oblk *b, int f, int x, int y, int z) {
  const box_t *q = &b->pbox[f];
  return (long)(x - q->x0) + (long)(q->x1 - q->x0 + 1) * ((long)(y - q->y0) + (long)(q->y1 - q->y0 + 1) * (long)(z - q->z0));
}

static double *zalloc(long n, double v) {
  double *p = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  for (long i = 0; i < n; ++i) p[i] = v;
  return p;
}

/* ------------------------------------------------------------------------ */
/* Grid and metrics: src/grid.f90:214-241 (cartesian_grid_3d),               */
/* src/grid.f90:398-471 (derivatives), src/metrics.f90:16-491 (D6x/y/z)      */
/* ------------------------------------------------------------------------ */
static void d6_line(const oblk *b, int axis, int x, int y, int z, double h, double out[3]) {
  int n = axis == 0 ? b->nx : axis == 1 ? b->ny : b->nz;
  int i = axis == 0 ? x : axis == 1 ? y : z;
  int cnt, idx[8];
  double c[8];
  sbp_stencil(i, n, &cnt, idx, c);
  for (int comp = 0; comp < 3; ++comp) {
    double s = 0.0;
    for (int k = 0; k < cnt; ++k) {
      int xx = axis == 0 ? idx[k] : x, yy = axis == 1 ? idx[k] : y, zz = axis == 2 ? idx[k] : z;
      double term = c[k] * b->X[comp][ID(b, xx, yy, zz)];
      s = (k == 0) ? term : s + term;
    }
    out[comp] = (1.0 / h) * s;   /* src/metrics.f90:166 */
  }
}

static void build_grid(oblk *b) {
  const orc_desc *d = &b->d;
  for (int c = 0; c < 3; ++c) b->X[c] = zalloc(b->np, 0.0);
  if (d->coords) {
    long n1 = (long)b->nx * b->ny * b->nz;
    for (int z = 1; z <= b->nz; ++z)
      for (int y = 1; y <= b->ny; ++y)
        for (int x = 1; x <= b->nx; ++x)
          for (int c = 0; c < 3; ++c)
            b->X[c][ID(b, x, y, z)] = d->coords[c * n1 + (x - 1) + (long)b->nx * ((y - 1) + (long)b->ny * (z - 1))];
  } else {
    double bh[3];
    int nn[3] = {b->nx, b->ny, b->nz};
    for (int c = 0; c < 3; ++c) bh[c] = (d->bqrs[c] - d->aqrs[c]) / (double)(nn[c] - 1);
    for (int z = 1; z <= b->nz; ++z)
      for (int y = 1; y <= b->ny; ++y)
        for (int x = 1; x <= b->nx; ++x) {
          long p = ID(b, x, y, z);
          b->X[0][p] = d->aqrs[0] + (double)(x - 1) * bh[0];
          b->X[1][p] = d->aqrs[1] + (double)(y - 1) * bh[1];
          b->X[2][p] = d->aqrs[2] + (double)(z - 1) * bh[2];
        }
  }
  b->hq = 1.0 / (double)(b->nx - 1);
  b->hr = 1.0 / (double)(b->ny - 1);
  b->hs = 1.0 / (double)(b->nz - 1);
  for (int c = 0; c < 3; ++c) { b->mx[c] = zalloc(b->np, 0.0); b->my[c] = zalloc(b->np, 0.0); b->mz[c] = zalloc(b->np, 0.0); }
  b->J = zalloc(b->np, 0.0);
  for (int s = 1; s <= b->nz; ++s)
    for (int r = 1; r <= b->ny; ++r)
      for (int q = 1; q <= b->nx; ++q) {
        double Xq[3], Xr[3], Xs[3];
        d6_line(b, 0, q, r, s, b->hq, Xq);
        d6_line(b, 1, q, r, s, b->hr, Xr);
        d6_line(b, 2, q, r, s, b->hs, Xs);
        long p = ID(b, q, r, s);
        double J = Xq[0] * (Xr[1] * Xs[2] - Xr[2] * Xs[1]) - Xq[1] * (Xr[0] * Xs[2] - Xr[2] * Xs[0]) +
                   Xq[2] * (Xr[0] * Xs[1] - Xr[1] * Xs[0]);
        b->J[p] = J;
        double iJ = 1.0 / J;
        b->mx[0][p] = iJ * (Xr[1] * Xs[2] - Xr[2] * Xs[1]);
        b->mx[1][p] = iJ * (Xq[2] * Xs[1] - Xq[1] * Xs[2]);
        b->mx[2][p] = iJ * (Xq[1] * Xr[2] - Xq[2] * Xr[1]);
        b->my[0][p] = iJ * (Xr[2] * Xs[0] - Xr[0] * Xs[2]);
        b->my[1][p] = iJ * (Xq[0] * Xs[2] - Xq[2] * Xs[0]);
        b->my[2][p] = iJ * (Xq[2] * Xr[0] - Xq[0] * Xr[2]);
        b->mz[0][p] = iJ * (Xr[0] * Xs[1] - Xr[1] * Xs[0]);
        b->mz[1][p] = iJ * (Xq[1] * Xs[0] - Xq[0] * Xs[1]);
        b->mz[2][p] = iJ * (Xq[0] * Xr[1] - Xq[1] * Xr[0]);
      }
}

/* ------------------------------------------------------------------------ */
/* Face normals: src/unit_normals.f90:8-266                                  */
/* ------------------------------------------------------------------------ */
static void gram_schmidt(const double y[3], double z[3]) { /* src/unit_normals.f90:252-264 */
  double a = y[0] * z[0] + y[1] * z[1] + y[2] * z[2];
  for (int i = 0; i < 3; ++i) z[i] = z[i] - a * y[i];
  double s = 1.0 / sqrt(z[0] * z[0] + z[1] * z[1] + z[2] * z[2]);
  for (int i = 0; i < 3; ++i) z[i] = s * z[i];
}

static void gen_orth(double l[3], double m[3], const double n[3]) { /* src/unit_normals.f90:217-249 */
  const double tol = 1.0e-12;
  m[0] = 0.0; m[1] = 1.0; m[2] = 0.0;
  double d1 = sqrt((n[0] - m[0]) * (n[0] - m[0]) + (n[1] - m[1]) * (n[1] - m[1]) + (n[2] - m[2]) * (n[2] - m[2]));
  double d2 = sqrt((n[0] + m[0]) * (n[0] + m[0]) + (n[1] + m[1]) * (n[1] + m[1]) + (n[2] + m[2]) * (n[2] + m[2]));
  if (!(d1 >= tol && d2 >= tol)) { m[0] = 0.0; m[1] = 0.0; m[2] = 1.0; }
  gram_schmidt(n, m);
  l[0] = n[1] * m[2] - n[2] * m[1];
  l[1] = n[2] * m[0] - n[0] * m[2];
  l[2] = n[0] * m[1] - n[1] * m[0];
}

static void build_normals(oblk *b) {
  for (int f = 0; f < 6; ++f) {
    int axis = f / 2;
    int d0 = axis == 0 ? b->ny : b->nx;
    int d1 = axis == 2 ? b->ny : b->nz;
    b->fdim[f][0] = d0; b->fdim[f][1] = d1;
    long n = (long)d0 * d1;
    for (int c = 0; c < 3; ++c) { b->nl[f][c] = zalloc(n, 0.0); b->nm[f][c] = zalloc(n, 0.0); b->nn[f][c] = zalloc(n, 0.0); }
    for (int c = 0; c < 9; ++c) b->work[f][c] = zalloc(n, 0.0);
    int fixed = (f % 2 == 0) ? 1 : (axis == 0 ? b->nx : axis == 1 ? b->ny : b->nz);
    for (int c2 = 1; c2 <= d1; ++c2)
      for (int c1 = 1; c1 <= d0; ++c1) {
        int x, y, z;
        if (axis == 0) { x = fixed; y = c1; z = c2; }
        else if (axis == 1) { x = c1; y = fixed; z = c2; }
        else { x = c1; y = c2; z = fixed; }
        long p = ID(b, x, y, z);
        double qx = b->mx[axis][p], qy = b->my[axis][p], qz = b->mz[axis][p];
        double norm = sqrt(qx * qx + qy * qy + qz * qz);
        double n3[3] = {qx / norm, qy / norm, qz / norm}, l3[3], m3[3];
        gen_orth(l3, m3, n3);
        long fp = FID(b, f, c1, c2);
        for (int c = 0; c < 3; ++c) { b->nn[f][c][fp] = n3[c]; b->nm[f][c][fp] = m3[c]; b->nl[f][c][fp] = l3[c]; }
      }
  }
}

/* ------------------------------------------------------------------------ */
/* Moment-tensor source: src/moment_tensor.f90:813-1125                      */
/* ------------------------------------------------------------------------ */
static double source_time(int type, double t, double t0, double w) {
  switch (type) {
    case ORC_STF_GAUSSIAN: return (w / (sqrt(2.0 * PI_WP))) * exp((-(w * w) * ((t - t0) * (t - t0))) / 2.0);
    case ORC_STF_LOH_DISC: return (t / (w * w)) * exp(-t / w);
    case ORC_STF_BRUNE: return (w * w) * t * exp(-w * t);
    case ORC_STF_COSBELL: return (t < t0) ? (1.0 - cos(2.0 * PI_WP * t / t0)) / t0 : 0.0;
    case ORC_STF_COSINE: return ((t >= 0.0) && (t <= w)) ? 1.0 - cos(2.0 * PI_WP * t / w) : 0.0;
    case ORC_STF_LOH_MOMENT: return (1.0 - (1.0 + t / w) * exp(-t / w));
    case ORC_STF_SINE_MOMENT: return (t <= w) ? t - w / (2.0 * PI_WP) * sin(2.0 * PI_WP * t / w) : w;
    case ORC_STF_RICKER: {
      /* Ricker wavelet, an addition (the reference has none): f0 = w, delay t0 */
      double a = PI_WP * w * (t - t0);
      double a2 = a * a;
      return (1.0 - 2.0 * a2) * exp(-a2);
    }
  }
  return 0.0;
}

static double singular_source(int i, int i0, double h, double a, int order, int alpha) {
  if (order == 2) { /* src/moment_tensor.f90:950-974 */
    double beta = (1.0 - 2.0 * a) / 4.0 + 0.25;
    double gam = (2.0 * a - 1.0) / 16.0;
    double gap = (2.0 * a + 1.0) / 16.0;
    if (i == i0 - 2) return (-gam) / h;
    if (i == i0 - 1) return (beta + 3.0 * gam - gap) / h;
    if (i == i0) return (1.0 - a - 2.0 * beta - 3.0 * gam + 3.0 * gap) / h;
    if (i == i0 + 1) return (a + beta + gam - 3.0 * gap) / h;
    if (i == i0 + 2) return gap / h;
    return 0.0;
  }
  if (order == 4) { /* src/moment_tensor.f90:976-1121 */
    static const double w0[9] = {-0.01171875, -0.03125, 0.046875, 0.28125, 0.4296875, 0.28125, 0.046875, -0.03125, -0.01171875};
    static const double w25[9] = {-0.00246875, -0.02275, -0.014125, 0.16575, 0.4171875, 0.38675, 0.117875, -0.02975, -0.01846875};
    static const double w50[9] = {-0.00728125, -0.028, 0.014875, 0.224, 0.4265625, 0.336, 0.081375, -0.032, -0.01553125};
    static const double w100[9] = {-0.0095625, -0.02990625, 0.03053125, 0.25284375, 0.42890625, 0.30903125, 0.06384375, -0.03196875, -0.01371875};
    const double *w = alpha == 0 ? w0 : alpha == 25 ? w25 : alpha == 50 ? w50 : alpha == 100 ? w100 : NULL;
    int k = i - i0;
    if (!w || k < -4 || k > 4) return 0.0;
    return w[k + 4] / h;
  }
  return 0.0;
}

/* Find_Coordinates_moment, src/seismogram.f90:878-960: nearest node, ties to the last visited */
static void nearest_node_moment(const oblk *b, double x1, double y1, double z1, int out[3]) {
  double mn[3] = {1e300, 1e300, 1e300}, mxv[3] = {-1e300, -1e300, -1e300};
  for (int z = 1; z <= b->nz; ++z)
    for (int y = 1; y <= b->ny; ++y)
      for (int x = 1; x <= b->nx; ++x)
        for (int c = 0; c < 3; ++c) {
          double v = b->X[c][ID(b, x, y, z)];
          if (v < mn[c]) mn[c] = v;
          if (v > mxv[c]) mxv[c] = v;
        }
  double scale = 1.0;
  for (int c = 0; c < 3; ++c) { if (fabs(mn[c]) > scale) scale = fabs(mn[c]); if (fabs(mxv[c]) > scale) scale = fabs(mxv[c]); }
  double tol = 1000.0 * 2.220446049250313e-16 * scale;
  out[0] = out[1] = out[2] = -9999;
  if (!((mn[0] - tol <= x1 && x1 <= mxv[0] + tol) && (mn[1] - tol <= y1 && y1 <= mxv[1] + tol) &&
        (mn[2] - tol <= z1 && z1 <= mxv[2] + tol)))
    return;
  double mindist = 1.0e8;
  for (int z = 1; z <= b->nz; ++z)
    for (int y = 1; y <= b->ny; ++y)
      for (int x = 1; x <= b->nx; ++x) {
        long p = ID(b, x, y, z);
        double v0 = b->X[0][p] - x1, v1 = b->X[1][p] - y1, v2 = b->X[2][p] - z1;
        double dist = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
        if (dist <= mindist) { out[0] = x; out[1] = y; out[2] = z; mindist = dist; }
      }
}

/* Find_Coordinates, src/seismogram.f90:767-876 (receivers) */
static void nearest_node_receiver(const oblk *b, double x1, double y1, double z1, int out[3]) {
  out[0] = out[1] = out[2] = -9999;
  double mindist = 1.0e8;
  int px = b->nx, py = b->ny, pz = b->nz;
  for (int k = 1; k <= pz; ++k)
    for (int j = 1; j <= py; ++j)
      for (int i = 1; i <= px; ++i) {
        double hx = b->X[0][ID(b, px, j, k)] - b->X[0][ID(b, px - 1, j, k)];
        double hy = b->X[1][ID(b, i, py, k)] - b->X[1][ID(b, i, py - 1, k)];
        double hz = b->X[2][ID(b, i, j, pz)] - b->X[2][ID(b, i, j, pz - 1)];
        if (i < px) hx = b->X[0][ID(b, i + 1, j, k)] - b->X[0][ID(b, i, j, k)];
        if (j < py) hy = b->X[1][ID(b, i, j + 1, k)] - b->X[1][ID(b, i, j, k)];
        if (k < pz) hz = b->X[2][ID(b, i, j, k + 1)] - b->X[2][ID(b, i, j, k)];
        long p = ID(b, i, j, k);
        double v0 = b->X[0][p] - x1, v1 = b->X[1][p] - y1, v2 = b->X[2][p] - z1;
        double dist = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
        double dist0 = sqrt(hx * hx + hy * hy + hz * hz);
        if ((dist <= mindist) && (dist <= 0.5 * dist0)) { out[0] = i; out[1] = j; out[2] = k; mindist = dist; }
      }
}

/* set_moment_tensor, src/moment_tensor.f90:875-936.  The reference visits
   every local point; the delta weights vanish outside the 5- or 9-point
   support, so only the support is visited here (exact: DF - A*M*0 = DF). */
static void set_moment_tensor(oblk *b, double t) {
  const orc_desc *d = &b->d;
  int half = d->src_order == 4 ? 4 : 2;
  for (int i = 0; i < b->nsrc; ++i) {
    const double *sp = &b->spar[i * 11];
    int nx0 = b->snear[3 * i], ny0 = b->snear[3 * i + 1], nz0 = b->snear[3 * i + 2];
    if (nx0 < 1) continue;
    double A = source_time(b->stype[i], t, sp[1], sp[0]);
    for (int n = nz0 - half; n <= nz0 + half; ++n) {
      if (n < 1 || n > b->nz) continue;
      for (int m = ny0 - half; m <= ny0 + half; ++m) {
        if (m < 1 || m > b->ny) continue;
        for (int l = nx0 - half; l <= nx0 + half; ++l) {
          if (l < 1 || l > b->nx) continue;
          long p = ID(b, l, m, n);
          double hx = b->hq / b->mx[0][p];
          double hy = b->hr / b->my[1][p];
          double hz = b->hs / b->mz[2][p];
          double ax = (sp[8] - b->sphys[3 * i]) / hx;
          double ay = (sp[9] - b->sphys[3 * i + 1]) / hy;
          double az = (sp[10] - b->sphys[3 * i + 2]) / hz;
          double dx = singular_source(l, nx0, hx, ax, d->src_order, d->src_alpha);
          double dy = singular_source(m, ny0, hy, ay, d->src_order, d->src_alpha);
          double dz = singular_source(n, nz0, hz, az, d->src_order, d->src_alpha);
          double delta = dx * dy * dz;
          b->DF[3][p] = b->DF[3][p] - A * sp[2] * delta;
          b->DF[4][p] = b->DF[4][p] - A * sp[3] * delta;
          b->DF[5][p] = b->DF[5][p] - A * sp[4] * delta;
          b->DF[6][p] = b->DF[6][p] - A * sp[5] * delta;
          b->DF[7][p] = b->DF[7][p] - A * sp[6] * delta;
          b->DF[8][p] = b->DF[8][p] - A * sp[7] * delta;
        }
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Near-boundary derivative JJU_x6, src/JU_xJU_yJU_z6.f90:12-809             */
/* X = metric row (metricx, metricy or metricz); components X[0..2] are the  */
/* q-, r-, s-entries of that row.                                            */
/* ------------------------------------------------------------------------ */
static void jju6(const oblk *b, int x, int y, int z, double *const X[3], double Ju[9]) {
  double Jq[9], Jr[9], Js[9];
  int cnt, idx[8];
  double c[8];
  long p0 = ID(b, x, y, z);
  /* q direction */
  sbp_stencil(x, b->nx, &cnt, idx, c);
  for (int f = 0; f < 9; ++f) {
    double s = 0.0;
    for (int k = 0; k < cnt; ++k) {
      long p = ID(b, idx[k], y, z);
      double term = f < 3 ? c[k] * b->F[f][p] : c[k] * b->F[f][p] * b->J[p] * X[0][p];
      s = (k == 0) ? term : s + term;
    }
    Jq[f] = f < 3 ? X[0][p0] * s : s;
  }
  sbp_stencil(y, b->ny, &cnt, idx, c);
  for (int f = 0; f < 9; ++f) {
    double s = 0.0;
    for (int k = 0; k < cnt; ++k) {
      long p = ID(b, x, idx[k], z);
      double term = f < 3 ? c[k] * b->F[f][p] : c[k] * b->F[f][p] * b->J[p] * X[1][p];
      s = (k == 0) ? term : s + term;
    }
    Jr[f] = f < 3 ? X[1][p0] * s : s;
  }
  sbp_stencil(z, b->nz, &cnt, idx, c);
  for (int f = 0; f < 9; ++f) {
    double s = 0.0;
    for (int k = 0; k < cnt; ++k) {
      long p = ID(b, x, y, idx[k]);
      double term = f < 3 ? c[k] * b->F[f][p] : c[k] * b->F[f][p] * b->J[p] * X[2][p];
      s = (k == 0) ? term : s + term;
    }
    Js[f] = f < 3 ? X[2][p0] * s : s;
  }
  for (int f = 0; f < 9; ++f) Ju[f] = (1.0 / b->hq) * Jq[f] + (1.0 / b->hr) * Jr[f] + (1.0 / b->hs) * Js[f];
}

/* ------------------------------------------------------------------------ */
/* Near-boundary upwind derivative (JJU_x4_upwind, JJU_x6_upwind,           */
/* JJU_x6_upwind_drp of src/JU_xJU_yJU_z6.f90): velocities X(p) * D+ u,      */
/* stresses D-((X J) F) with the reference's association ((c X) J) F of each */
/* term.                                                                     */
/* ------------------------------------------------------------------------ */
static void jju_up(const oblk *b, const upwind_op *op, int x, int y, int z, double *const X[3], double Ju[9]) {
  double Jd[3][9];
  int cnt, idx[UP_MAXT];
  double c[UP_MAXT];
  const long p0 = ID(b, x, y, z);
  const int pos[3] = {x, y, z}, nn[3] = {b->nx, b->ny, b->nz};
  for (int a = 0; a < 3; ++a) {
    for (int plus = 1; plus >= 0; --plus) {
      up_stencil(op, plus, pos[a], nn[a], &cnt, idx, c);
      for (int f = plus ? 0 : 3; f < (plus ? 3 : 9); ++f) {
        double s = 0.0;
        for (int k = 0; k < cnt; ++k) {
          const int q[3] = {a == 0 ? idx[k] : x, a == 1 ? idx[k] : y, a == 2 ? idx[k] : z};
          const long p = ID(b, q[0], q[1], q[2]);
          const double term = plus ? c[k] * b->F[f][p] : c[k] * X[a][p] * b->J[p] * b->F[f][p];
          s = (k == 0) ? term : s + term;
        }
        Jd[a][f] = plus ? X[a][p0] * s : s;
      }
    }
  }
  for (int f = 0; f < 9; ++f) Ju[f] = (1.0 / b->hq) * Jd[0][f] + (1.0 / b->hr) * Jd[1][f] + (1.0 / b->hs) * Jd[2][f];
}

/* ------------------------------------------------------------------------ */
/* PML: src/RHS_Interior.f90:1846-2265, src/RHS_Interior.f90:2351-2451       */
/* ------------------------------------------------------------------------ */
static double pml_d0(void) { return 6.0 / (2.0 * 1.0) * log(1.0 / 1.0e-3); }

static int in_slab(const oblk *b, int f, int x, int y, int z) {
  const box_t *q = &b->pbox[f];
  if (!q->active) return 0;
  return x >= q->x0 && x <= q->x1 && y >= q->y0 && y <= q->y1 && z >= q->z0 && z <= q->z1;
}

/* damping for face f (0-based) at the point's coordinate */
static double pml_damp(const oblk *b, int f, int x, int y, int z) {
  int np = b->d.npml;
  double d0 = pml_d0();
  double v;
  switch (f) {
    case 0: v = (double)(x - (1 + np)); break;
    case 1: v = (double)(x - (b->nx - np)); break;
    case 2: v = (double)(y - (1 + np)); break;
    case 3: v = (double)(y - (b->ny - np)); break;
    case 4: v = (double)(z - np); break;        /* asymmetric offset, src/RHS_Interior.f90:1919 */
    default: v = (double)(z - (b->nz - np)); break;
  }
  return d0 * fabs(v / (double)np);
}

static void pml_point(oblk *b, double DU[9], const double Ux[9], const double Uy[9], const double Uz[9],
                      int x, int y, int z, double rhoJ_inv, double lambda2mu) {
  static const int order[6] = {4, 5, 2, 3, 0, 1}; /* the reference applies z, y, x slabs in this order */
  long p = ID(b, x, y, z);
  double lam = b->M[0][p], mu = b->M[1][p];
  double J = b->J[p];
  const double cfs = 1.0;
  for (int oi = 0; oi < 6; ++oi) {
    int f = order[oi];
    if (!b->d.pml[f] || !b->pbox[f].active) continue;
    if (!in_slab(b, f, x, y, z)) continue;
    double d = pml_damp(b, f, x, y, z);
    long q = PID(b, f, x, y, z);
    double *Qf[9], *DQf[9];
    for (int c = 0; c < 9; ++c) { Qf[c] = b->Q[f][c]; DQf[c] = b->DQ[f][c]; }
    DU[0] = DU[0] - d * J * Qf[0][q] * rhoJ_inv;
    DU[1] = DU[1] - d * J * Qf[1][q] * rhoJ_inv;
    DU[2] = DU[2] - d * J * Qf[2][q] * rhoJ_inv;
    DU[3] = DU[3] - d * (lambda2mu * Qf[3][q] + lam * Qf[4][q] + lam * Qf[5][q]);
    DU[4] = DU[4] - d * (lam * Qf[3][q] + lambda2mu * Qf[4][q] + lam * Qf[5][q]);
    DU[5] = DU[5] - d * (lam * Qf[3][q] + lam * Qf[4][q] + lambda2mu * Qf[5][q]);
    DU[6] = DU[6] - mu * d * Qf[6][q];
    DU[7] = DU[7] - mu * d * Qf[7][q];
    DU[8] = DU[8] - mu * d * Qf[8][q];
    double src[9];
    int axis = f / 2;
    if (axis == 2) { /* z slabs, src/RHS_Interior.f90:1936-1962 */
      src[0] = Uz[7] / J; src[1] = Uz[8] / J; src[2] = Uz[5] / J; src[3] = 0.0; src[4] = 0.0;
      src[5] = Uz[2]; src[6] = 0.0; src[7] = Uz[0]; src[8] = Uz[1];
    } else if (axis == 1) { /* y slabs */
      src[0] = Uy[6] / J; src[1] = Uy[4] / J; src[2] = Uy[8] / J; src[3] = 0.0; src[4] = Uy[1];
      src[5] = 0.0; src[6] = Uy[0]; src[7] = 0.0; src[8] = Uy[2];
    } else { /* x slabs */
      src[0] = Ux[3] / J; src[1] = Ux[6] / J; src[2] = Ux[7] / J; src[3] = Ux[0]; src[4] = 0.0;
      src[5] = 0.0; src[6] = Ux[1]; src[7] = Ux[2]; src[8] = 0.0;
    }
    for (int c = 0; c < 9; ++c) DQf[c][q] = DQf[c][q] + src[c] - (d + cfs) * Qf[c][q];
  }
}

/* pml_damping_and_q, src/RHS_Interior.f90:2351-2451 */
static int pml_damping_and_q(const oblk *b, int x, int y, int z, double *dx, double *dy, double *dz,
                             double Qx[9], double Qy[9], double Qz[9]) {
  int inpml = 0;
  *dx = *dy = *dz = 0.0;
  for (int c = 0; c < 9; ++c) Qx[c] = Qy[c] = Qz[c] = 0.0;
  for (int f = 0; f < 6; ++f) {
    if (!b->d.pml[f] || !b->pbox[f].active || !in_slab(b, f, x, y, z)) continue;
    inpml = 1;
    double d = pml_damp(b, f, x, y, z);
    long q = PID(b, f, x, y, z);
    double *dd = f < 2 ? dx : f < 4 ? dy : dz;
    double *QQ = f < 2 ? Qx : f < 4 ? Qy : Qz;
    *dd = d;
    for (int c = 0; c < 9; ++c) QQ[c] = b->Q[f][c][q];
  }
  return inpml;
}

/* ------------------------------------------------------------------------ */
/* Anelastic memory variables (Q4 / Q8 / fQ8):                               */
/* src/RHS_Interior.f90:2599-2908 (Q4, Q8 point kernels + PML variants),     */
/* src/RHS_Interior.f90:3361-3477 (fQ8), interior copies                     */
/* src/JU_xJU_yJU_z6.f90:16263-16420.                                        */
/* exx..gyz are the (PML-corrected) strain rates.                            */
/* ------------------------------------------------------------------------ */
static void anelastic_point(oblk *b, long p, int x, int y, int z, double exx, double eyy, double ezz,
                            double gxy, double gxz, double gyz, double tr, double DU[9], int dfmode) {
  int N = b->nmech;
  double lam = b->M[0][p], mu = b->M[1][p];
  double sum[6];
  for (int c = 0; c < 6; ++c) {
    double s = b->eta[c][0][p];
    for (int i = 1; i < N; ++i) s = s + b->eta[c][i][p];
    sum[c] = s;
  }
  if (dfmode) {
    for (int c = 0; c < 6; ++c) b->DF[3 + c][p] = b->DF[3 + c][p] - sum[c];
  } else {
    for (int c = 0; c < 6; ++c) DU[3 + c] = DU[3 + c] - sum[c];
  }
  double e_n[3] = {exx, eyy, ezz};
  double g_s[3] = {gxy, gxz, gyz};
  if (b->d.response == ORC_FQ8) {
    int active = 1 + ((x - 1) % 2) + 2 * ((y - 1) % 2) + 4 * ((z - 1) % 2);
    for (int i = 0; i < N; ++i) {
      if (b->d.coarse && (i + 1) != active) continue;
      double ss = b->d.sstr[i], ps = b->d.pstr[i], tau = b->d.tau[i];
      for (int c = 0; c < 3; ++c) {
        double *De = &b->deta[c][i][p];
        *De = *De + (((ss * 2.0 * mu) * e_n[c] + ((lam + 2.0 * mu) * ps - 2.0 * mu * ss) * tr) - b->eta[c][i][p]) / tau;
      }
      for (int c = 0; c < 3; ++c) {
        double *De = &b->deta[3 + c][i][p];
        *De = *De + ((ss * mu * g_s[c] - b->eta[3 + c][i][p]) / tau);
      }
    }
  } else {
    double qs = b->qs[p], qp = b->qp[p];
    for (int i = 0; i < N; ++i) {
      double w = b->d.weight[i], tau = b->d.tau[i];
      for (int c = 0; c < 3; ++c) {
        double *De = &b->deta[c][i][p];
        *De = *De + (((w * 2.0 * mu * qs) * e_n[c] + (w * ((lam + 2.0 * mu) * qp - 2.0 * mu * qs)) * tr) - b->eta[c][i][p]) / tau;
      }
      for (int c = 0; c < 3; ++c) {
        double *De = &b->deta[3 + c][i][p];
        *De = *De + ((w * mu * qs * g_s[c] - b->eta[3 + c][i][p]) / tau);
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* RHS_near_boundaries (traditional branch), src/RHS_Interior.f90:136-281    */
/* ------------------------------------------------------------------------ */
static void interior_bounds(const oblk *b, int lo[3], int hi[3]) {
  /* src/RHS_Interior.f90:199-214, src/JU_xJU_yJU_z6.f90:16158-16173; the
     upwind widths: 4 for upwind-4 (src/JU_xJU_yJU_z6.f90:17915-17931), 6 for
     upwind-6, 8 for upwind-DRP-6 (src/RHS_Interior.f90:614-630, 1218-1234) */
  const upwind_op *op = upwind_of(b->d.fd);
  const int w = op ? op->width : 6;
  int ix = w, iy = w, iz = w, fx = w, fy = w, fz = w;
  const int *pm = b->d.pml;
  int np = b->d.npml;
  if (pm[4]) iz = np > w ? np : w;
  if (pm[5]) fz = np > w ? np : w;
  if (pm[2]) iy = np > w ? np : w;
  if (pm[3]) fy = np > w ? np : w;
  if (pm[0]) ix = np > w ? np : w;
  if (pm[1]) fx = np > w ? np : w;
  lo[0] = ix + 1; hi[0] = b->nx - fx;
  lo[1] = iy + 1; hi[1] = b->ny - fy;
  lo[2] = iz + 1; hi[2] = b->nz - fz;
}

static void rhs_near_boundaries(oblk *b) {
  int lo[3], hi[3];
  interior_bounds(b, lo, hi);
  const upwind_op *op = upwind_of(b->d.fd);
#pragma omp parallel for schedule(static)
  for (int z = 1; z <= b->nz; ++z)
    for (int y = 1; y <= b->ny; ++y)
      for (int x = 1; x <= b->nx; ++x) {
        if ((lo[2] <= z && z <= hi[2]) && (lo[1] <= y && y <= hi[1]) && (lo[0] <= x && x <= hi[0])) continue;
        double Ux[9], Uy[9], Uz[9], DU[9];
        if (op) { /* src/RHS_Interior.f90:443-470, 614-660, 1218-1260 */
          jju_up(b, op, x, y, z, b->mx, Ux);
          jju_up(b, op, x, y, z, b->my, Uy);
          jju_up(b, op, x, y, z, b->mz, Uz);
        } else {
          jju6(b, x, y, z, b->mx, Ux);
          jju6(b, x, y, z, b->my, Uy);
          jju6(b, x, y, z, b->mz, Uz);
        }
        long p = ID(b, x, y, z);
        double rhoJ_inv = 1.0 / (b->M[2][p] * b->J[p]);
        double lambda2mu = b->M[0][p] + 2.0 * b->M[1][p];
        double lam = b->M[0][p], mu = b->M[1][p];
        DU[0] = (Ux[3] + Uy[6] + Uz[7]) * rhoJ_inv;
        DU[1] = (Ux[6] + Uy[4] + Uz[8]) * rhoJ_inv;
        DU[2] = (Ux[7] + Uy[8] + Uz[5]) * rhoJ_inv;
        DU[3] = lambda2mu * Ux[0] + lam * (Uy[1] + Uz[2]);
        DU[4] = lambda2mu * Uy[1] + lam * (Ux[0] + Uz[2]);
        DU[5] = lambda2mu * Uz[2] + lam * (Ux[0] + Uy[1]);
        DU[6] = mu * (Uy[0] + Ux[1]);
        DU[7] = mu * (Uz[0] + Ux[2]);
        DU[8] = mu * (Uz[1] + Uy[2]);
        if (b->d.response != ORC_ELASTIC) {
          /* apply_anelastic_*_point_dispatch: PML variant corrects the strain rates */
          double dxp, dyp, dzp, Qx[9], Qy[9], Qz[9];
          double exx, eyy, ezz, gxy, gxz, gyz, tr;
          if (pml_damping_and_q(b, x, y, z, &dxp, &dyp, &dzp, Qx, Qy, Qz)) {
            exx = Ux[0] - dxp * Qx[3];
            eyy = Uy[1] - dyp * Qy[4];
            ezz = Uz[2] - dzp * Qz[5];
            tr = exx + eyy + ezz;
            gxy = (Uy[0] + Ux[1]) - dxp * Qx[6] - dyp * Qy[6];
            gxz = (Uz[0] + Ux[2]) - dxp * Qx[7] - dzp * Qz[7];
            gyz = (Uz[1] + Uy[2]) - dyp * Qy[8] - dzp * Qz[8];
          } else {
            exx = Ux[0]; eyy = Uy[1]; ezz = Uz[2];
            tr = Ux[0] + Uy[1] + Uz[2];
            gxy = Uy[0] + Ux[1]; gxz = Uz[0] + Ux[2]; gyz = Uz[1] + Uy[2];
          }
          anelastic_point(b, p, x, y, z, exx, eyy, ezz, gxy, gxz, gyz, tr, DU, 0);
        }
        pml_point(b, DU, Ux, Uy, Uz, x, y, z, rhoJ_inv, lambda2mu);
        for (int f = 0; f < 9; ++f) b->DF[f][p] = b->DF[f][p] + DU[f];
      }
}

/* ------------------------------------------------------------------------ */
/* Strict interior JJU_x6_interior, src/JU_xJU_yJU_z6.f90:16088-16640        */
/* ------------------------------------------------------------------------ */
/* Rates of a strict-interior point from its derivative terms, shared by both
   interior routines (src/JU_xJU_yJU_z6.f90:16426-16636, :17990-18120). */
static void interior_rates(oblk *b, long p, int x, int y, int z, int curv, const double DFx[9],
                           const double DFy[9], const double DFz[9]) {
  double a1 = curv ? 1.0 / (b->M[2][p] * b->J[p]) : 1.0 / b->M[2][p];
  double a2 = 2.0 * b->M[1][p] + b->M[0][p];
  double a3 = b->M[0][p];
  double a4 = b->M[1][p];
  b->DF[0][p] = b->DF[0][p] + a1 * (DFx[3] + DFy[6] + DFz[7]);
  b->DF[1][p] = b->DF[1][p] + a1 * (DFx[6] + DFy[4] + DFz[8]);
  b->DF[2][p] = b->DF[2][p] + a1 * (DFx[7] + DFy[8] + DFz[5]);
  b->DF[3][p] = b->DF[3][p] + a2 * DFx[0] + a3 * (DFy[1] + DFz[2]);
  b->DF[4][p] = b->DF[4][p] + a2 * DFy[1] + a3 * (DFx[0] + DFz[2]);
  b->DF[5][p] = b->DF[5][p] + a2 * DFz[2] + a3 * (DFx[0] + DFy[1]);
  b->DF[6][p] = b->DF[6][p] + a4 * (DFy[0] + DFx[1]);
  b->DF[7][p] = b->DF[7][p] + a4 * (DFz[0] + DFx[2]);
  b->DF[8][p] = b->DF[8][p] + a4 * (DFz[1] + DFy[2]);
  if (b->d.response != ORC_ELASTIC) {
    double tr = DFx[0] + DFy[1] + DFz[2];
    anelastic_point(b, p, x, y, z, DFx[0], DFy[1], DFz[2], DFy[0] + DFx[1], DFz[0] + DFx[2], DFz[1] + DFy[2], tr,
                    NULL, 1);
  }
}

/* ------------------------------------------------------------------------ */
/* Strict interior of the upwind operators (JJU_x4_interior_upwind,         */
/* src/JU_xJU_yJU_z6.f90:17865-18400; JJU_x6_interior_upwind, :18958-19510;  */
/* JJU_x6_interior_upwind_drp): forward differences of the velocities at     */
/* offsets of .. of + taps - 1, backward differences of the stresses at      */
/* ob .. ob + taps - 1; Cartesian: diagonal metric at the point, 1/rho;      */
/* curvilinear: metric at the point for the velocities, (F X) J at the taps  */
/* for the stresses.                                                         */
/* ------------------------------------------------------------------------ */
static void rhs_interior_up(oblk *b, const upwind_op *op) {
  int lo[3], hi[3];
  interior_bounds(b, lo, hi);
  const int T = op->taps;
  double cfx[10], cfy[10], cfz[10], cbx[10], cby[10], cbz[10];
  for (int k = 0; k < T; ++k) {
    cfx[k] = op->inf_[k] / b->hq; cfy[k] = op->inf_[k] / b->hr; cfz[k] = op->inf_[k] / b->hs;
    cbx[k] = op->inb[k] / b->hq; cby[k] = op->inb[k] / b->hr; cbz[k] = op->inb[k] / b->hs;
  }
  const long sx = 1, sy = b->NX, sz = (long)b->NX * b->NY;
  const int curv = b->d.mesh == 1;
#pragma omp parallel for schedule(static)
  for (int z = lo[2]; z <= hi[2]; ++z)
    for (int y = lo[1]; y <= hi[1]; ++y)
      for (int x = lo[0]; x <= hi[0]; ++x) {
        const long p = ID(b, x, y, z);
        double DFx[9] = {0}, DFy[9] = {0}, DFz[9] = {0};
        for (int k = 0; k < T; ++k) {
          const long s = op->of + k, t = op->ob + k;
          const long fx = p + s * sx, fy = p + s * sy, fz = p + s * sz;  /* forward taps */
          const long bx = p + t * sx, by = p + t * sy, bz = p + t * sz;  /* backward taps */
          if (curv) {
            for (int f = 0; f < 3; ++f) {
              const double *Ff = b->F[f];
              DFx[f] = DFx[f] + b->mx[0][p] * cfx[k] * Ff[fx] + b->mx[1][p] * cfy[k] * Ff[fy] + b->mx[2][p] * cfz[k] * Ff[fz];
              DFy[f] = DFy[f] + b->my[0][p] * cfx[k] * Ff[fx] + b->my[1][p] * cfy[k] * Ff[fy] + b->my[2][p] * cfz[k] * Ff[fz];
              DFz[f] = DFz[f] + b->mz[0][p] * cfx[k] * Ff[fx] + b->mz[1][p] * cfy[k] * Ff[fy] + b->mz[2][p] * cfz[k] * Ff[fz];
            }
            for (int f = 3; f < 9; ++f) {
              const double *Ff = b->F[f];
              DFx[f] = DFx[f] + cbx[k] * Ff[bx] * b->mx[0][bx] * b->J[bx] + cby[k] * Ff[by] * b->mx[1][by] * b->J[by] +
                       cbz[k] * Ff[bz] * b->mx[2][bz] * b->J[bz];
              DFy[f] = DFy[f] + cbx[k] * Ff[bx] * b->my[0][bx] * b->J[bx] + cby[k] * Ff[by] * b->my[1][by] * b->J[by] +
                       cbz[k] * Ff[bz] * b->my[2][bz] * b->J[bz];
              DFz[f] = DFz[f] + cbx[k] * Ff[bx] * b->mz[0][bx] * b->J[bx] + cby[k] * Ff[by] * b->mz[1][by] * b->J[by] +
                       cbz[k] * Ff[bz] * b->mz[2][bz] * b->J[bz];
            }
          } else {
            for (int f = 0; f < 3; ++f) {
              DFx[f] = DFx[f] + b->mx[0][p] * cfx[k] * b->F[f][fx];
              DFy[f] = DFy[f] + b->my[1][p] * cfy[k] * b->F[f][fy];
              DFz[f] = DFz[f] + b->mz[2][p] * cfz[k] * b->F[f][fz];
            }
            for (int f = 3; f < 9; ++f) {
              DFx[f] = DFx[f] + b->mx[0][p] * cbx[k] * b->F[f][bx];
              DFy[f] = DFy[f] + b->my[1][p] * cby[k] * b->F[f][by];
              DFz[f] = DFz[f] + b->mz[2][p] * cbz[k] * b->F[f][bz];
            }
          }
        }
        interior_rates(b, p, x, y, z, curv, DFx, DFy, DFz);
      }
}

static void rhs_interior(oblk *b) {
  if (upwind_of(b->d.fd)) {
    rhs_interior_up(b, upwind_of(b->d.fd));
    return;
  }
  int lo[3], hi[3];
  interior_bounds(b, lo, hi);
  static const double c[3] = {0.75, -0.15, 1.0 / 60.0};
  double cx[3], cy[3], cz[3];
  for (int s = 0; s < 3; ++s) { cx[s] = c[s] / b->hq; cy[s] = c[s] / b->hr; cz[s] = c[s] / b->hs; }
  const long sx = 1, sy = b->NX, sz = (long)b->NX * b->NY;
  int curv = b->d.mesh == 1;
#pragma omp parallel for schedule(static)
  for (int z = lo[2]; z <= hi[2]; ++z)
    for (int y = lo[1]; y <= hi[1]; ++y)
      for (int x = lo[0]; x <= hi[0]; ++x) {
        long p = ID(b, x, y, z);
        double DFx[9] = {0}, DFy[9] = {0}, DFz[9] = {0};
        if (curv) { /* :16177-16424 */
          for (int s = 1; s <= 3; ++s) {
            double ccx = cx[s - 1], ccy = cy[s - 1], ccz = cz[s - 1];
            long xp = p + s * sx, xm = p - s * sx, yp = p + s * sy, ym = p - s * sy, zp = p + s * sz, zm = p - s * sz;
            for (int f = 0; f < 3; ++f) {
              double ddx = b->F[f][xp] - b->F[f][xm], ddy = b->F[f][yp] - b->F[f][ym], ddz = b->F[f][zp] - b->F[f][zm];
              DFx[f] = DFx[f] + b->mx[0][p] * ccx * ddx + b->mx[1][p] * ccy * ddy + b->mx[2][p] * ccz * ddz;
              DFy[f] = DFy[f] + b->my[0][p] * ccx * ddx + b->my[1][p] * ccy * ddy + b->my[2][p] * ccz * ddz;
              DFz[f] = DFz[f] + b->mz[0][p] * ccx * ddx + b->mz[1][p] * ccy * ddy + b->mz[2][p] * ccz * ddz;
            }
            for (int f = 3; f < 9; ++f) {
              const double *Ff = b->F[f];
              DFx[f] = DFx[f] + ccx * (Ff[xp] * (b->J[xp] * b->mx[0][xp]) - Ff[xm] * (b->J[xm] * b->mx[0][xm])) +
                       ccy * (Ff[yp] * (b->J[yp] * b->mx[1][yp]) - Ff[ym] * (b->J[ym] * b->mx[1][ym])) +
                       ccz * (Ff[zp] * (b->J[zp] * b->mx[2][zp]) - Ff[zm] * (b->J[zm] * b->mx[2][zm]));
              DFy[f] = DFy[f] + ccx * (Ff[xp] * (b->J[xp] * b->my[0][xp]) - Ff[xm] * (b->J[xm] * b->my[0][xm])) +
                       ccy * (Ff[yp] * (b->J[yp] * b->my[1][yp]) - Ff[ym] * (b->J[ym] * b->my[1][ym])) +
                       ccz * (Ff[zp] * (b->J[zp] * b->my[2][zp]) - Ff[zm] * (b->J[zm] * b->my[2][zm]));
              DFz[f] = DFz[f] + ccx * (Ff[xp] * (b->J[xp] * b->mz[0][xp]) - Ff[xm] * (b->J[xm] * b->mz[0][xm])) +
                       ccy * (Ff[yp] * (b->J[yp] * b->mz[1][yp]) - Ff[ym] * (b->J[ym] * b->mz[1][ym])) +
                       ccz * (Ff[zp] * (b->J[zp] * b->mz[2][zp]) - Ff[zm] * (b->J[zm] * b->mz[2][zm]));
            }
          }
        } else { /* Cartesian, :16426-16450 */
          for (int s = 1; s <= 3; ++s)
            for (int f = 0; f < 9; ++f) {
              DFx[f] = DFx[f] + b->mx[0][p] * cx[s - 1] * (b->F[f][p + s * sx] - b->F[f][p - s * sx]);
              DFy[f] = DFy[f] + b->my[1][p] * cy[s - 1] * (b->F[f][p + s * sy] - b->F[f][p - s * sy]);
              DFz[f] = DFz[f] + b->mz[2][p] * cz[s - 1] * (b->F[f][p + s * sz] - b->F[f][p - s * sz]);
            }
        }
        interior_rates(b, p, x, y, z, curv, DFx, DFy, DFz);
      }
}

/* ------------------------------------------------------------------------ */
/* Physical-boundary SAT: src/BoundaryConditions.f90:50-924,                 */
/* src/RHS_Interior.f90:1584-1768 (impose), :2267-2287 (structure)           */
/* ------------------------------------------------------------------------ */
static void bc_point(int plus, const double u[9], double rho, double mu, double lambda, const double l[3],
                     const double m[3], const double n[3], double norm, double Zs, double Zp, double r,
                     double ubc[9]) {
  double T[3];
  T[0] = n[0] * u[3] + n[1] * u[6] + n[2] * u[7];
  T[1] = n[0] * u[6] + n[1] * u[4] + n[2] * u[8];
  T[2] = n[0] * u[7] + n[1] * u[8] + n[2] * u[5];
  double vl = l[0] * u[0] + l[1] * u[1] + l[2] * u[2];
  double vm = m[0] * u[0] + m[1] * u[1] + m[2] * u[2];
  double vn = n[0] * u[0] + n[1] * u[1] + n[2] * u[2];
  double Tl = l[0] * T[0] + l[1] * T[1] + l[2] * T[2];
  double Tm = m[0] * T[0] + m[1] * T[1] + m[2] * T[2];
  double Tn = n[0] * T[0] + n[1] * T[1] + n[2] * T[2];
  double pl, pm, pn, ql, qm, qn;
  if (plus) { /* BCp, :783-852 */
    pl = 0.5 * ((1.0 - r) * Zs * vl + (1.0 + r) * Tl);
    pm = 0.5 * ((1.0 - r) * Zs * vm + (1.0 + r) * Tm);
    pn = 0.5 * ((1.0 - r) * Zp * vn + (1.0 + r) * Tn);
    ql = 0.5 * ((1.0 - r) * vl + (1.0 + r) / Zs * Tl);
    qm = 0.5 * ((1.0 - r) * vm + (1.0 + r) / Zs * Tm);
    qn = 0.5 * ((1.0 - r) * vn + (1.0 + r) / Zp * Tn);
  } else { /* BCm, :855-924 */
    pl = 0.5 * ((1.0 - r) * Zs * vl - (1.0 + r) * Tl);
    pm = 0.5 * ((1.0 - r) * Zs * vm - (1.0 + r) * Tm);
    pn = 0.5 * ((1.0 - r) * Zp * vn - (1.0 + r) * Tn);
    ql = 0.5 * ((1.0 - r) * vl - (1.0 + r) / Zs * Tl);
    qm = 0.5 * ((1.0 - r) * vm - (1.0 + r) / Zs * Tm);
    qn = 0.5 * ((1.0 - r) * vn - (1.0 + r) / Zp * Tn);
  }
  double Fx = l[0] * pl + m[0] * pm + n[0] * pn;
  double Fy = l[1] * pl + m[1] * pm + n[1] * pn;
  double Fz = l[2] * pl + m[2] * pm + n[2] * pn;
  double F_x = l[0] * ql + m[0] * qm + n[0] * qn;
  double F_y = l[1] * ql + m[1] * qm + n[1] * qn;
  double F_z = l[2] * ql + m[2] * qm + n[2] * qn;
  (void)rho; (void)mu; (void)lambda;
  double sg = plus ? 1.0 : -1.0;
  ubc[0] = norm * Fx;
  ubc[1] = norm * Fy;
  ubc[2] = norm * Fz;
  ubc[3] = sg * (norm * n[0] * F_x);
  ubc[4] = sg * (norm * n[1] * F_y);
  ubc[5] = sg * (norm * n[2] * F_z);
  ubc[6] = sg * (norm * (n[1] * F_x + n[0] * F_y));
  ubc[7] = sg * (norm * (n[2] * F_x + n[0] * F_z));
  ubc[8] = sg * (norm * (n[2] * F_y + n[1] * F_z));
}

static void structure(double Ux[9], const double Uq[9], double rho, double mu, double lam) {
  Ux[0] = 1.0 / rho * Uq[0];
  Ux[1] = 1.0 / rho * Uq[1];
  Ux[2] = 1.0 / rho * Uq[2];
  Ux[3] = (2.0 * mu + lam) * Uq[3] + lam * (Uq[4] + Uq[5]);
  Ux[4] = (2.0 * mu + lam) * Uq[4] + lam * (Uq[3] + Uq[5]);
  Ux[5] = (2.0 * mu + lam) * Uq[5] + lam * (Uq[3] + Uq[4]);
  Ux[6] = mu * Uq[6];
  Ux[7] = mu * Uq[7];
  Ux[8] = mu * Uq[8];
}

/* ------------------------------------------------------------------------ */
/* Manufactured solution: src/mms.f90:136-235                                */
/* ------------------------------------------------------------------------ */
static void mms_eval(const orc_desc *d, double t, const double X[3], double u[9]) {
  const double ct = cos(d->mms_nt * PI_WP * t);
  const double a = sin(d->mms_nx * PI_WP * X[0]) * sin(d->mms_ny * PI_WP * X[1]) * sin(d->mms_nz * PI_WP * X[2]);
  const double c = cos(d->mms_nx * PI_WP * X[0]) * cos(d->mms_ny * PI_WP * X[1]) * cos(d->mms_nz * PI_WP * X[2]);
  for (int k = 0; k < 3; ++k) u[k] = ct * a;
  for (int k = 3; k < 9; ++k) u[k] = ct * c;
}

/* time and space derivatives of the solution, :176-235 */
static void mms_derivs(const orc_desc *d, double t, const double X[3], double ut[9], double ux[9], double uy[9],
                       double uz[9]) {
  const double kt = d->mms_nt * PI_WP, kx = d->mms_nx * PI_WP, ky = d->mms_ny * PI_WP, kz = d->mms_nz * PI_WP;
  const double ct = cos(kt * t), st = sin(kt * t);
  const double sx = sin(kx * X[0]), cx = cos(kx * X[0]);
  const double sy = sin(ky * X[1]), cy = cos(ky * X[1]);
  const double sz = sin(kz * X[2]), cz = cos(kz * X[2]);
  for (int k = 0; k < 3; ++k) {
    ut[k] = -kt * st * sx * sy * sz;
    ux[k] = kx * ct * cx * sy * sz;
    uy[k] = ky * ct * sx * cy * sz;
    uz[k] = kz * ct * sx * sy * cz;
  }
  for (int k = 3; k < 9; ++k) {
    ut[k] = -kt * st * cx * cy * cz;
    ux[k] = -kx * ct * sx * cy * cz;
    uy[k] = -ky * ct * cx * sy * cz;
    uz[k] = -kz * ct * cx * cy * sz;
  }
}

/* DU -= L(u*) - u*_t at every point (mms_forcing, src/mms.f90:77-134) */
static void mms_forcing(oblk *b, double t) {
  for (int z = 1; z <= b->nz; ++z)
    for (int y = 1; y <= b->ny; ++y)
      for (int x = 1; x <= b->nx; ++x) {
        long p = ID(b, x, y, z);
        double X[3] = {b->X[0][p], b->X[1][p], b->X[2][p]};
        double ut[9], ux[9], uy[9], uz[9], f[9];
        mms_derivs(&b->d, t, X, ut, ux, uy, uz);
        const double lam = b->M[0][p], mu = b->M[1][p], rho = b->M[2][p];
        f[0] = (1.0 / rho) * (ux[3] + uy[6] + uz[7]);
        f[1] = (1.0 / rho) * (ux[6] + uy[4] + uz[8]);
        f[2] = (1.0 / rho) * (ux[7] + uy[8] + uz[5]);
        f[3] = (2.0 * mu + lam) * ux[0] + lam * uy[1] + lam * uz[2];
        f[4] = lam * ux[0] + (2.0 * mu + lam) * uy[1] + lam * uz[2];
        f[5] = lam * ux[0] + lam * uy[1] + (2.0 * mu + lam) * uz[2];
        f[6] = mu * (uy[0] + ux[1]);
        f[7] = mu * (uz[0] + ux[2]);
        f[8] = mu * (uz[1] + uy[2]);
        for (int c = 0; c < 9; ++c) b->DF[c][p] = b->DF[c][p] - (f[c] - ut[c]);
      }
}

static void impose_boundary_condition(oblk *b, double t) {
  const double tau0 = b->d.tau0;
  const double hs_[3] = {b->hq, b->hr, b->hs};
  for (int f = 0; f < 6; ++f) {
    int type = b->d.bc[f];
    if (type <= 0) continue;
    int axis = f / 2, plus = f % 2;
    double r = type == 1 ? 0.0 : type == 2 ? 1.0 : -1.0;
    int fixed = plus ? (axis == 0 ? b->nx : axis == 1 ? b->ny : b->nz) : 1;
    int d0 = b->fdim[f][0], d1 = b->fdim[f][1];
    /* BC_* builds u_bc for the whole face first, then impose applies it */
    for (int c2 = 1; c2 <= d1; ++c2)
      for (int c1 = 1; c1 <= d0; ++c1) {
        int x, y, z;
        if (axis == 0) { x = fixed; y = c1; z = c2; }
        else if (axis == 1) { x = c1; y = fixed; z = c2; }
        else { x = c1; y = c2; z = fixed; }
        long p = ID(b, x, y, z);
        double rho = b->M[2][p], mu = b->M[1][p], lambda = b->M[0][p];
        double c_p = sqrt((2.0 * mu + lambda) / rho);
        double c_s = sqrt(mu / rho);
        double Zp = rho * c_p, Zs = rho * c_s;
        double qx = b->mx[axis][p], qy = b->my[axis][p], qz = b->mz[axis][p];
        double norm = sqrt(qx * qx + qy * qy + qz * qz);
        long fp = FID(b, f, c1, c2);
        double l3[3], m3[3], n3[3], u[9], ubc[9];
        for (int c = 0; c < 3; ++c) { l3[c] = b->nl[f][c][fp]; m3[c] = b->nm[f][c][fp]; n3[c] = b->nn[f][c][fp]; }
        for (int c = 0; c < 9; ++c) u[c] = b->F[c][p];
        if (b->d.mms) { /* u - switch*fu, src/BoundaryConditions.f90:84-88 */
          double X[3] = {b->X[0][p], b->X[1][p], b->X[2][p]}, fu[9];
          mms_eval(&b->d, t, X, fu);
          for (int c = 0; c < 9; ++c) u[c] = u[c] - 1.0 * fu[c];
        }
        bc_point(plus, u, rho, mu, lambda, l3, m3, n3, norm, Zs, Zp, r, ubc);
        for (int c = 0; c < 9; ++c) b->work[f][c][fp] = ubc[c];
      }
    double h = hs_[axis];
    for (int c2 = 1; c2 <= d1; ++c2)
      for (int c1 = 1; c1 <= d0; ++c1) {
        int x, y, z;
        if (axis == 0) { x = fixed; y = c1; z = c2; }
        else if (axis == 1) { x = c1; y = fixed; z = c2; }
        else { x = c1; y = c2; z = fixed; }
        long p = ID(b, x, y, z);
        long fp = FID(b, f, c1, c2);
        double Uq[9], Ux[9];
        for (int c = 0; c < 9; ++c) Uq[c] = b->work[f][c][fp];
        structure(Ux, Uq, b->M[2][p], b->M[1][p], b->M[0][p]);
        for (int c = 0; c < 9; ++c) b->DF[c][p] = b->DF[c][p] - tau0 / h * Ux[c];
        if (b->d.pml[f] && b->pbox[f].active && in_slab(b, f, x, y, z)) {
          long q = PID(b, f, x, y, z);
          for (int c = 0; c < 9; ++c) b->DQ[f][c][q] = b->DQ[f][c][q] - tau0 / h * Uq[c];
        }
      }
  }
}

/* ------------------------------------------------------------------------ */
/* Block-interface coupling (q direction): src/CouplingForcing.f90:9-463,     */
/* src/Interface_Condition.f90:12-916                                         */
/* ------------------------------------------------------------------------ */
void orc_iface_couple(odom *D, int ib, double t, int stage);

/* ------------------------------------------------------------------------ */
/* Block creation                                                            */
/* ------------------------------------------------------------------------ */
static oblk *block_create(const orc_desc *d) {
  sbp_init(d->f32lit);
  oblk *b = (oblk *)calloc(1, sizeof(oblk));
  b->d = *d;
  b->nx = d->nq; b->ny = d->nr; b->nz = d->ns;
  b->NX = b->nx + 2 * NB; b->NY = b->ny + 2 * NB; b->NZ = b->nz + 2 * NB;
  b->np = (long)b->NX * b->NY * b->NZ;
  build_grid(b);
  long n1 = (long)b->nx * b->ny * b->nz;
  for (int c = 0; c < 3; ++c) b->M[c] = zalloc(b->np, 0.0);
  for (int z = 1; z <= b->nz; ++z)
    for (int y = 1; y <= b->ny; ++y)
      for (int x = 1; x <= b->nx; ++x) {
        long p = ID(b, x, y, z);
        long q = (x - 1) + (long)b->nx * ((y - 1) + (long)b->ny * (z - 1));
        if (d->material) {
          for (int c = 0; c < 3; ++c) b->M[c][p] = d->material[c * n1 + q];
        } else { /* src/material.f90:696-701 */
          const double *r = d->rho_s_p;
          b->M[0][p] = r[0] * (r[2] * r[2] - 2.0 * (r[1] * r[1]));
          b->M[1][p] = r[0] * (r[1] * r[1]);
          b->M[2][p] = r[0];
        }
      }
  for (int c = 0; c < 9; ++c) { b->F[c] = zalloc(b->np, 0.0); b->DF[c] = zalloc(b->np, 1.0e40); } /* src/fields.f90:38-39 */
  /* PML slabs, src/pml.f90:11-168 */
  for (int f = 0; f < 6; ++f) {
    box_t *q = &b->pbox[f];
    q->x0 = 1; q->x1 = b->nx; q->y0 = 1; q->y1 = b->ny; q->z0 = 1; q->z1 = b->nz;
    q->active = d->pml[f] && d->npml > 0;
    if (!q->active) continue;
    int np = d->npml;
    switch (f) {
      case 0: q->x1 = np; break;
      case 1: q->x0 = b->nx - np + 1; break;
      case 2: q->y1 = np; break;
      case 3: q->y0 = b->ny - np + 1; break;
      case 4: q->z1 = np; break;
      default: q->z0 = b->nz - np + 1; break;
    }
    long n = (long)(q->x1 - q->x0 + 1) * (q->y1 - q->y0 + 1) * (q->z1 - q->z0 + 1);
    for (int c = 0; c < 9; ++c) { b->Q[f][c] = zalloc(n, 0.0); b->DQ[f][c] = zalloc(n, 1.0e40); }
  }
  /* anelastic state */
  if (d->response != ORC_ELASTIC) {
    b->nmech = d->response == ORC_Q4 ? 4 : 8;
    b->qs = zalloc(b->np, 0.0);
    b->qp = zalloc(b->np, 0.0);
    for (int z = 1; z <= b->nz; ++z)
      for (int y = 1; y <= b->ny; ++y)
        for (int x = 1; x <= b->nx; ++x) {
          long p = ID(b, x, y, z);
          long q = (x - 1) + (long)b->nx * ((y - 1) + (long)b->ny * (z - 1));
          if (d->qsinv) b->qs[p] = d->qsinv[q];
          if (d->qpinv) b->qp[p] = d->qpinv[q];
        }
    for (int c = 0; c < 6; ++c)
      for (int i = 0; i < b->nmech; ++i) { b->eta[c][i] = zalloc(b->np, 0.0); b->deta[c][i] = zalloc(b->np, 0.0); }
  }
  build_normals(b);
  /* sources */
  b->nsrc = d->nsrc;
  if (b->nsrc > 0) {
    b->stype = (int *)malloc(sizeof(int) * b->nsrc);
    b->spar = (double *)malloc(sizeof(double) * 11 * b->nsrc);
    b->snear = (int *)malloc(sizeof(int) * 3 * b->nsrc);
    b->sphys = (double *)malloc(sizeof(double) * 3 * b->nsrc);
    memcpy(b->stype, d->src_type, sizeof(int) * b->nsrc);
    memcpy(b->spar, d->src_par, sizeof(double) * 11 * b->nsrc);
    for (int i = 0; i < b->nsrc; ++i) {
      nearest_node_moment(b, b->spar[11 * i + 8], b->spar[11 * i + 9], b->spar[11 * i + 10], &b->snear[3 * i]);
      if (b->snear[3 * i] > 0) {
        long p = ID(b, b->snear[3 * i], b->snear[3 * i + 1], b->snear[3 * i + 2]);
        for (int c = 0; c < 3; ++c) b->sphys[3 * i + c] = b->X[c][p];
      } else {
        for (int c = 0; c < 3; ++c) b->sphys[3 * i + c] = -1.0;
      }
    }
  }
  b->nrec = d->nrec;
  if (b->nrec > 0) {
    b->ridx = (int *)malloc(sizeof(int) * 3 * b->nrec);
    for (int i = 0; i < b->nrec; ++i)
      nearest_node_receiver(b, d->rec_xyz[3 * i], d->rec_xyz[3 * i + 1], d->rec_xyz[3 * i + 2], &b->ridx[3 * i]);
  }
  for (int s = 0; s < 2; ++s) {
    long n = (long)b->ny * b->nz;
    for (int c = 0; c < 9; ++c) { b->faceF[s][c] = zalloc(n, 0.0); b->faceFopp[s][c] = zalloc(n, 0.0); }
    for (int c = 0; c < 3; ++c) { b->faceM[s][c] = zalloc(n, 0.0); b->faceMopp[s][c] = zalloc(n, 0.0); }
  }
  /* copy_materials_to_boundary, src/block.f90:484-495 */
  for (int z = 1; z <= b->nz; ++z)
    for (int y = 1; y <= b->ny; ++y) {
      long fp = (y - 1) + (long)b->ny * (z - 1);
      for (int c = 0; c < 3; ++c) {
        b->faceM[0][c][fp] = b->M[c][ID(b, 1, y, z)];
        b->faceM[1][c][fp] = b->M[c][ID(b, b->nx, y, z)];
      }
    }
  return b;
}

static void block_free(oblk *b) {
  if (!b) return;
  for (int c = 0; c < 3; ++c) { free(b->X[c]); free(b->mx[c]); free(b->my[c]); free(b->mz[c]); free(b->M[c]); }
  free(b->J);
  for (int c = 0; c < 9; ++c) { free(b->F[c]); free(b->DF[c]); }
  for (int f = 0; f < 6; ++f) {
    for (int c = 0; c < 9; ++c) { free(b->Q[f][c]); free(b->DQ[f][c]); free(b->work[f][c]); }
    for (int c = 0; c < 3; ++c) { free(b->nl[f][c]); free(b->nm[f][c]); free(b->nn[f][c]); }
  }
  free(b->qs); free(b->qp);
  for (int c = 0; c < 6; ++c)
    for (int i = 0; i < 8; ++i) { free(b->eta[c][i]); free(b->deta[c][i]); }
  free(b->stype); free(b->spar); free(b->snear); free(b->sphys); free(b->ridx);
  for (int s = 0; s < 2; ++s) {
    for (int c = 0; c < 9; ++c) { free(b->faceF[s][c]); free(b->faceFopp[s][c]); }
    for (int c = 0; c < 3; ++c) { free(b->faceM[s][c]); free(b->faceMopp[s][c]); }
  }
  free(b);
}

/* ------------------------------------------------------------------------ */
/* RK vector operations: src/rk_vector_cpu.f90:7-18, fan-out                 */
/* src/fields.f90:51-263                                                     */
/* ------------------------------------------------------------------------ */
static void scale_rates_block(oblk *b, double A) {
  for (int c = 0; c < 9; ++c)
    for (long i = 0; i < b->np; ++i) b->DF[c][i] = A * b->DF[c][i];
  for (int c = 0; c < 6; ++c)
    for (int k = 0; k < b->nmech; ++k)
      for (long i = 0; i < b->np; ++i) b->deta[c][k][i] = A * b->deta[c][k][i];
  for (int f = 0; f < 6; ++f) {
    if (!b->pbox[f].active) continue;
    const box_t *q = &b->pbox[f];
    long n = (long)(q->x1 - q->x0 + 1) * (q->y1 - q->y0 + 1) * (q->z1 - q->z0 + 1);
    for (int c = 0; c < 9; ++c)
      for (long i = 0; i < n; ++i) b->DQ[f][c][i] = A * b->DQ[f][c][i];
  }
}

static void update_fields_block(oblk *b, double dt) {
  for (int c = 0; c < 9; ++c)
    for (long i = 0; i < b->np; ++i) b->F[c][i] = b->F[c][i] + dt * b->DF[c][i];
  for (int c = 0; c < 6; ++c)
    for (int k = 0; k < b->nmech; ++k)
      for (long i = 0; i < b->np; ++i) b->eta[c][k][i] = b->eta[c][k][i] + dt * b->deta[c][k][i];
  for (int f = 0; f < 6; ++f) {
    if (!b->pbox[f].active) continue;
    const box_t *q = &b->pbox[f];
    long n = (long)(q->x1 - q->x0 + 1) * (q->y1 - q->y0 + 1) * (q->z1 - q->z0 + 1);
    for (int c = 0; c < 9; ++c)
      for (long i = 0; i < n; ++i) b->Q[f][c][i] = b->Q[f][c][i] + dt * b->DQ[f][c][i];
  }
}

/* ------------------------------------------------------------------------ */
/* Low-storage RK: src/time_step.f90:20-150 (Kennedy-Carpenter (5,4))        */
/* ------------------------------------------------------------------------ */
static const double RK_A[5] = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                               -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
static const double RK_B[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                               1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                               2277821191437.0 / 14882151754819.0};
static const double RK_C[6] = {0.0, 1432997174477.0 / 9575080441755.0, 2526269341429.0 / 6820363962896.0,
                               2006345519317.0 / 3224310063776.0, 2802321613138.0 / 2924317926251.0, 1.0};

static void iface_scale(oiface *I, double A) {
  if (!I) return;
  long n = (long)I->nr * I->ns;
  for (int c = 0; c < 4; ++c)
    for (long i = 0; i < n; ++i) I->DS[c][i] = A * I->DS[c][i];
  for (long i = 0; i < n; ++i) I->DW[i] = A * I->DW[i];
}

static void iface_update(oiface *I, double dt) {
  if (!I) return;
  long n = (long)I->nr * I->ns;
  for (int c = 0; c < 4; ++c)
    for (long i = 0; i < n; ++i) I->S[c][i] = I->S[c][i] + dt * I->DS[c][i];
  for (long i = 0; i < n; ++i) I->W[i] = I->W[i] + dt * I->DW[i];
}

static void copy_fields_to_boundary(oblk *b) { /* src/block.f90:466-482 */
  for (int c = 0; c < 9; ++c)
    for (int z = 1; z <= b->nz; ++z)
      for (int y = 1; y <= b->ny; ++y) {
        long fp = (y - 1) + (long)b->ny * (z - 1);
        b->faceF[0][c][fp] = b->F[c][ID(b, 1, y, z)];
        b->faceF[1][c][fp] = b->F[c][ID(b, b->nx, y, z)];
      }
}

static void sample_receivers(oblk *b, double t, double *out) {
  for (int r = 0; r < b->nrec; ++r) {
    int i = b->ridx[3 * r], j = b->ridx[3 * r + 1], k = b->ridx[3 * r + 2];
    out[4 * r] = t;
    if (i > 0 && j > 0 && k > 0) {
      long p = ID(b, i, j, k);
      out[4 * r + 1] = b->F[0][p]; out[4 * r + 2] = b->F[1][p]; out[4 * r + 3] = b->F[2][p];
    } else {
      out[4 * r + 1] = out[4 * r + 2] = out[4 * r + 3] = 0.0;
    }
  }
}

static void do_stage(odom *D, int stage, double dt, double t0, int sample, double *seis0, double *seis1) {
  /* exchange_fields: single rank, no-op */
  for (int i = 0; i < D->nb; ++i) scale_rates_block(D->B[i], RK_A[stage - 1]);
  iface_scale(D->I, RK_A[stage - 1]);
  for (int i = 0; i < D->nb; ++i) {
    oblk *b = D->B[i];
    rhs_interior(b);
    rhs_near_boundaries(b);
    if (b->nsrc > 0) set_moment_tensor(b, D->t);
    if (b->d.mms) mms_forcing(b, D->t);
  }
  if (D->nb == 2) { /* exchange_fields_interface, src/domain.f90:696-726 (serial copy) */
    copy_fields_to_boundary(D->B[0]);
    copy_fields_to_boundary(D->B[1]);
    long n = (long)D->B[0]->ny * D->B[0]->nz;
    for (int c = 0; c < 9; ++c)
      for (long k = 0; k < n; ++k) {
        D->B[0]->faceFopp[1][c][k] = D->B[1]->faceF[0][c][k];
        D->B[1]->faceFopp[0][c][k] = D->B[0]->faceF[1][c][k];
      }
  }
  /* enforce_bound_iface_conditions, src/domain.f90:615-644 */
  impose_boundary_condition(D->B[0], D->t);
  if (D->nb == 2) orc_iface_couple(D, 2, D->t, stage);
  if (D->nb == 2) {
    impose_boundary_condition(D->B[1], D->t);
    orc_iface_couple(D, 1, D->t, stage);
  }
  if (sample) {
    if (seis0) sample_receivers(D->B[0], D->t, seis0);
    if (seis1 && D->nb == 2) sample_receivers(D->B[1], D->t, seis1);
  }
  D->t = t0 + RK_C[stage] * dt;
  for (int i = 0; i < D->nb; ++i) update_fields_block(D->B[i], RK_B[stage - 1] * dt);
  iface_update(D->I, RK_B[stage - 1] * dt);
}

/* ------------------------------------------------------------------------ */
/* Public API                                                                */
/* ------------------------------------------------------------------------ */
static void rs_init_vel_state(odom *D);

void *orc_create(int nblocks, const orc_desc *blocks, const orc_iface_desc *iface) {
  odom *D = (odom *)calloc(1, sizeof(odom));
  D->nb = nblocks;
  for (int i = 0; i < nblocks; ++i) D->B[i] = block_create(&blocks[i]);
  if (nblocks == 2) {
    oblk *b0 = D->B[0], *b1 = D->B[1];
    long n = (long)b0->ny * b0->nz;
    for (int c = 0; c < 3; ++c)
      for (long k = 0; k < n; ++k) { /* exchange_materials_interface, src/domain.f90:728-754 */
        b0->faceMopp[1][c][k] = b1->faceM[0][c][k];
        b1->faceMopp[0][c][k] = b0->faceM[1][c][k];
      }
    oiface *I = (oiface *)calloc(1, sizeof(oiface));
    if (iface) I->d = *iface;
    I->nr = b0->ny; I->ns = b0->nz;
    for (int c = 0; c < 4; ++c) { I->S[c] = zalloc(n, 0.0); I->DS[c] = zalloc(n, 0.0); }
    I->W = zalloc(n, 0.0); I->DW = zalloc(n, 0.0);
    for (int c = 0; c < 3; ++c) I->Svel[c] = zalloc(n, 0.0);
    for (int c = 0; c < 6; ++c) { I->Uhat[c] = zalloc(n, 0.0); I->Vhat[c] = zalloc(n, 0.0); }
    I->trup = zalloc(n, 1.0e9);
    I->t0n = zalloc(n, 0.0); I->t0m = zalloc(n, 0.0); I->t0l = zalloc(n, 0.0); I->fsm = zalloc(n, iface ? iface->fs : 0.0);
    if (iface) {
      for (long k = 0; k < n; ++k) {
        if (iface->tau0_n) I->t0n[k] = iface->tau0_n[k];
        if (iface->tau0_m) I->t0m[k] = iface->tau0_m[k];
        if (iface->tau0_l) I->t0l[k] = iface->tau0_l[k];
        if (iface->fs_map) I->fsm[k] = iface->fs_map[k];
      }
    }
    D->I = I;
    if (I->d.coupling == ORC_IFACE_RATE_STATE) rs_init_vel_state(D);
  }
  D->t = 0.0;
  return D;
}

void orc_destroy(void *dv) {
  odom *D = (odom *)dv;
  if (!D) return;
  for (int i = 0; i < D->nb; ++i) block_free(D->B[i]);
  if (D->I) {
    for (int c = 0; c < 4; ++c) { free(D->I->S[c]); free(D->I->DS[c]); }
    for (int c = 0; c < 3; ++c) free(D->I->Svel[c]);
    for (int c = 0; c < 6; ++c) { free(D->I->Uhat[c]); free(D->I->Vhat[c]); }
    free(D->I->W); free(D->I->DW); free(D->I->trup);
    free(D->I->t0n); free(D->I->t0m); free(D->I->t0l); free(D->I->fsm);
    free(D->I);
  }
  free(D);
}

double orc_time(void *dv) { return ((odom *)dv)->t; }
void orc_set_time(void *dv, double t) { ((odom *)dv)->t = t; }

int orc_run(void *dv, double dt, int nsteps, int w_stride, double *seis0, double *seis1) {
  odom *D = (odom *)dv;
  int nsamp = 0;
  for (int n = 1; n <= nsteps; ++n) {
    double t0 = D->t;
    int sample = (w_stride > 0) && ((n - 1) % w_stride == 0);
    double *s0 = (sample && seis0) ? seis0 + (long)nsamp * 4 * D->B[0]->nrec : NULL;
    double *s1 = (sample && seis1 && D->nb == 2) ? seis1 + (long)nsamp * 4 * D->B[1]->nrec : NULL;
    for (int stage = 1; stage <= 5; ++stage) do_stage(D, stage, dt, t0, stage == 1 && sample, s0, s1);
    if (sample) ++nsamp;
  }
  return nsamp;
}

void orc_stage(void *dv, int stage, double dt) {
  odom *D = (odom *)dv;
  do_stage(D, stage, dt, D->t, 0, NULL, NULL);
}

static void get3(const oblk *b, double *const *src, int ncomp, double *out) {
  long n1 = (long)b->nx * b->ny * b->nz;
  for (int c = 0; c < ncomp; ++c)
    for (int z = 1; z <= b->nz; ++z)
      for (int y = 1; y <= b->ny; ++y)
        for (int x = 1; x <= b->nx; ++x)
          out[c * n1 + (x - 1) + (long)b->nx * ((y - 1) + (long)b->ny * (z - 1))] = src[c][ID(b, x, y, z)];
}
static void set3(oblk *b, double *const *dst, int ncomp, const double *in) {
  long n1 = (long)b->nx * b->ny * b->nz;
  for (int c = 0; c < ncomp; ++c)
    for (int z = 1; z <= b->nz; ++z)
      for (int y = 1; y <= b->ny; ++y)
        for (int x = 1; x <= b->nx; ++x)
          dst[c][ID(b, x, y, z)] = in[c * n1 + (x - 1) + (long)b->nx * ((y - 1) + (long)b->ny * (z - 1))];
}

void orc_get_fields(void *dv, int bi, double *out) { oblk *b = ((odom *)dv)->B[bi]; get3(b, b->F, 9, out); }
void orc_set_fields(void *dv, int bi, const double *in) { oblk *b = ((odom *)dv)->B[bi]; set3(b, b->F, 9, in); }
void orc_get_rates(void *dv, int bi, double *out) { oblk *b = ((odom *)dv)->B[bi]; get3(b, b->DF, 9, out); }
void orc_set_rates(void *dv, int bi, const double *in) { oblk *b = ((odom *)dv)->B[bi]; set3(b, b->DF, 9, in); }
void orc_get_material(void *dv, int bi, double *out) { oblk *b = ((odom *)dv)->B[bi]; get3(b, b->M, 3, out); }
void orc_get_metrics(void *dv, int bi, double *out) {
  oblk *b = ((odom *)dv)->B[bi];
  double *arr[10] = {b->mx[0], b->mx[1], b->mx[2], b->my[0], b->my[1], b->my[2], b->mz[0], b->mz[1], b->mz[2], b->J};
  get3(b, arr, 10, out);
}
int orc_get_eta(void *dv, int bi, double *out) {
  oblk *b = ((odom *)dv)->B[bi];
  long n1 = (long)b->nx * b->ny * b->nz;
  for (int c = 0; c < 6; ++c) get3(b, b->eta[c], b->nmech, out + (long)c * b->nmech * n1);
  return b->nmech;
}
void orc_set_eta(void *dv, int bi, const double *in) {
  oblk *b = ((odom *)dv)->B[bi];
  long n1 = (long)b->nx * b->ny * b->nz;
  for (int c = 0; c < 6; ++c) set3(b, b->eta[c], b->nmech, in + (long)c * b->nmech * n1);
}
void orc_get_pml(void *dv, int bi, int face, double *out) {
  oblk *b = ((odom *)dv)->B[bi];
  const box_t *q = &b->pbox[face];
  if (!q->active) return;
  long n = (long)(q->x1 - q->x0 + 1) * (q->y1 - q->y0 + 1) * (q->z1 - q->z0 + 1);
  for (int c = 0; c < 9; ++c) memcpy(out + c * n, b->Q[face][c], sizeof(double) * n);
}
void orc_get_normals(void *dv, int bi, int face, double *out) {
  oblk *b = ((odom *)dv)->B[bi];
  long n = (long)b->fdim[face][0] * b->fdim[face][1];
  for (int c = 0; c < 3; ++c) {
    memcpy(out + (0 + c) * n, b->nl[face][c], sizeof(double) * n);
    memcpy(out + (3 + c) * n, b->nm[face][c], sizeof(double) * n);
    memcpy(out + (6 + c) * n, b->nn[face][c], sizeof(double) * n);
  }
}
void orc_get_iface(void *dv, double *out) {
  odom *D = (odom *)dv;
  if (!D->I) return;
  long n = (long)D->I->nr * D->I->ns;
  for (long k = 0; k < n; ++k) {
    for (int c = 0; c < 4; ++c) out[7 * k + c] = D->I->S[c][k];
    out[7 * k + 4] = D->I->W[k];
    out[7 * k + 5] = sqrt(D->I->Svel[1][k] * D->I->Svel[1][k] + D->I->Svel[2][k] * D->I->Svel[2][k]);
    out[7 * k + 6] = D->I->trup[k];
  }
}
void orc_mms_exact(void *dv, int bi, double t, double *out) {
  oblk *b = ((odom *)dv)->B[bi];
  long n1 = (long)b->nx * b->ny * b->nz;
  for (int z = 1; z <= b->nz; ++z)
    for (int y = 1; y <= b->ny; ++y)
      for (int x = 1; x <= b->nx; ++x) {
        long p = ID(b, x, y, z);
        double X[3] = {b->X[0][p], b->X[1][p], b->X[2][p]}, u[9];
        mms_eval(&b->d, t, X, u);
        long q = (x - 1) + (long)b->nx * ((y - 1) + (long)b->ny * (z - 1));
        for (int c = 0; c < 9; ++c) out[c * n1 + q] = u[c];
      }
}
void orc_receiver_index(void *dv, int bi, int *idx) {
  oblk *b = ((odom *)dv)->B[bi];
  memcpy(idx, b->ridx, sizeof(int) * 3 * b->nrec);
}

/* close_domain diagnostics, src/domain.f90:505-613: max over the whole
   allocated arrays (ghost layers included) */
void orc_final_state(void *dv, double *maxF, double *maxEta, double *maxB) {
  odom *D = (odom *)dv;
  double mf = 0.0, me = 0.0;
  for (int i = 0; i < D->nb; ++i) {
    oblk *b = D->B[i];
    double mb = 0.0;
    for (int c = 0; c < 9; ++c)
      for (long k = 0; k < b->np; ++k) { double v = fabs(b->F[c][k]); if (v > mb) mb = v; }
    if (maxB) maxB[i] = mb;
    if (mb > mf) mf = mb;
    for (int c = 0; c < 6; ++c)
      for (int m = 0; m < b->nmech; ++m)
        for (long k = 0; k < b->np; ++k) { double v = fabs(b->eta[c][m][k]); if (v > me) me = v; }
  }
  *maxF = mf;
  *maxEta = me;
}

/* Row of an upwind operator (ORC_FD_UPWIND*; plus = 1: D+, 0: D-) at 1-based
   i of n points: up to 13 (1-based index, coefficient) pairs; returns the
   count, 0 for a traditional-6 code */
int orc_upwind_row(int fd, int plus, int i, int n, int *idx, double *c) {
  const upwind_op *op = upwind_of(fd);
  if (!op) return 0;
  int cnt = 0;
  up_stencil(op, plus, i, n, &cnt, idx, c);
  return cnt;
}

/* Q4 / Q8 fixed coefficients */
void orc_q4_coefficients(double fmin, double fmax, double *tau, double *weight) {
  double taumin = 1.0 / (2.0 * PI_WP * fmax), taumax = 1.0 / (2.0 * PI_WP * fmin);
  for (int k = 1; k <= 4; ++k) tau[k - 1] = exp(log(taumin) + (2.0 * k - 1.0) / (2.0 * 4) * log(taumax / taumin));
  static const double w[4] = {1.549360, 0.804277, 0.887718, 1.464160};
  memcpy(weight, w, sizeof(w));
}
void orc_q8_coefficients(double fmin, double fmax, double *tau, double *weight) {
  double taumin = 1.0 / (2.0 * PI_WP * fmax), taumax = 1.0 / (2.0 * PI_WP * fmin);
  for (int k = 1; k <= 8; ++k) tau[k - 1] = exp(log(taumin) + (2.0 * k - 1.0) / (2.0 * 8) * log(taumax / taumin));
  static const double w[8] = {1.50589707, 0.0, 0.52793567, 0.53065494, 0.32862132, 0.64375916, 0.0, 1.32751442};
  memcpy(weight, w, sizeof(w));
}
void orc_modulus_correction(int nmech, const double *tau, const double *weight, double fref, long n, double *lam,
                            double *mu, const double *rho, const double *qsinv, const double *qpinv) {
  double wref = 2.0 * PI_WP * fref;
  for (long i = 0; i < n; ++i) {
    double vS = 0.0, vP = 0.0;
    for (int l = 0; l < nmech; ++l) {
      double dS = ((wref * wref) * (tau[l] * tau[l]) + 1.0) * (1.0 / qsinv[i]);
      double dP = ((wref * wref) * (tau[l] * tau[l]) + 1.0) * (1.0 / qpinv[i]);
      vS = vS + weight[l] / dS;
      vP = vP + weight[l] / dP;
    }
    double vs = sqrt(mu[i] / rho[i]);
    double vp = sqrt((lam[i] + 2.0 * mu[i]) / rho[i]);
    double muS = rho[i] * (vs * vs) / (1.0 - vS);
    double muP = rho[i] * (vp * vp) / (1.0 - vP);
    vs = sqrt(muS / rho[i]);
    vp = sqrt(muP / rho[i]);
    mu[i] = (vs * vs) * rho[i];
    lam[i] = (vp * vp) * rho[i] - 2.0 * mu[i];
  }
}

/* ------------------------------------------------------------------------ */
/* Block-interface coupling (q direction)                                    */
/* ------------------------------------------------------------------------ */

/* boxcar of unit amplitude on (-w, w), 1/2 within 100 eps of the edges:
   src/Interface_Condition.f90:2438-2457 */
static double boxcar(double x, double w) {
  const double tol = 100.0 * 2.220446049250313e-16;
  if (-w + tol < x && x < w - tol) return 1.0;
  if (fabs(-w - x) <= tol || fabs(x - w) <= tol) return 0.5;
  return 0.0;
}

/* initial tractions on the fault: src/Interface_Condition.f90:1802-1830 (TPV5),
   :2049-2076 with src/initial_stress_condition.f90:78-84 (TPV28: the uniform
   stress tensor projected on the point's (n, m, l) basis plus the nucleation
   shear), or the per-point maps of the description */
static void fault_prestress(const oiface *I, long k, const double x[3], const double n[3], const double m[3],
                            const double l[3], double *T0n, double *T0m, double *T0l) {
  if (I->d.problem == ORC_FAULT_TPV28) {
    static const double tpv28[6] = {-60.0, 0.0, 60.0, 0.0, 29.38, 0.0};
    const double *s0 = tpv28;
    for (int c = 0; c < 6; ++c)
      if (I->d.s0[c] != 0.0) s0 = I->d.s0;
    const double sxx = s0[0], syy = s0[1], szz = s0[2], sxy = s0[3], sxz = s0[4], syz = s0[5];
    const double Tx = n[0] * sxx + n[1] * sxy + n[2] * sxz;
    const double Ty = n[0] * sxy + n[1] * syy + n[2] * syz;
    const double Tz = n[0] * sxz + n[1] * syz + n[2] * szz;
    *T0n = n[0] * Tx + n[1] * Ty + n[2] * Tz;
    *T0m = m[0] * Tx + m[1] * Ty + m[2] * Tz;
    *T0l = l[0] * Tx + l[1] * Ty + l[2] * Tz;
    const double r = sqrt((x[1] - 7.5) * (x[1] - 7.5) + x[2] * x[2]);
    double nuke = 0.0;
    if (r <= 1.4) nuke = 11.60;
    else if (r >= 1.4 && r <= 2.0) nuke = 5.8 * (1.0 + cos(PI_WP * (r - 1.4) / 0.6));
    *T0l = *T0l + nuke;
    return;
  }
  if (I->d.problem == ORC_FAULT_TPV5) {
    double tl = 70.0;
    tl = tl + 8.0 * boxcar(x[1] - 7.5, 1.5) * boxcar(x[2] + 7.5, 1.5);
    tl = tl + 11.6 * boxcar(x[1] - 7.5, 1.5) * boxcar(x[2], 1.5);
    tl = tl - 8.0 * boxcar(x[1] - 7.5, 1.5) * boxcar(x[2] - 7.5, 1.5);
    *T0n = -120.0; *T0m = 0.0; *T0l = tl;
    return;
  }
  *T0n = I->t0n[k]; *T0m = I->t0m[k]; *T0l = I->t0l[k];
}

/* fault strength tau_str = sigma_n * f(slip): src/Interface_Condition.f90:1268-1299 */
static double fault_strength(const oiface *I, long k, const double x[3], double sigma_n, double D) {
  double fs, fd, Dc;
  if (I->d.problem == ORC_FAULT_TPV5) {
    fs = 0.677; fd = 0.525; Dc = 0.4;
    fs = fs + 1.0e10 * (1.0 - boxcar(x[1], 15.0) * boxcar(x[2], 15.0));
  } else if (I->d.problem == ORC_FAULT_TPV28) { /* src/Interface_Condition.f90:1459-1474 */
    fs = 0.677; fd = 0.373; Dc = 0.4;
    fs = fs + 1.0e10 * (1.0 - boxcar(x[1], 15.0) * boxcar(x[2], 18.0));
  } else {
    fs = I->fsm[k]; fd = I->d.fd; Dc = I->d.Dc;
  }
  double f = fs - (fs - fd) * fmin(D, Dc) / Dc;
  return sigma_n * f;
}

/* characteristic variables p = Z1 u - T (side 1), q = Z2 v + T (side 2) and the
   locked-interface flux phi: common head of Welded_Interface, Linear_Friction and
   Slip_Weakening_Friction (src/Interface_Condition.f90:540-575, 660-690, 780-815) */
typedef struct {
  double p[3], q[3], phi[3], eta_p, eta_s;
} char_t;

static void characteristics(const double *U, const double *V, double Z1s, double Z2s, double Z1p, double Z2p,
                            char_t *c) {
  c->p[0] = Z1p * U[0] - U[3];
  c->p[1] = Z1s * U[1] - U[4];
  c->p[2] = Z1s * U[2] - U[5];
  c->q[0] = Z2p * V[0] + V[3];
  c->q[1] = Z2s * V[1] + V[4];
  c->q[2] = Z2s * V[2] + V[5];
  c->eta_p = 1.0 / (1.0 / Z1p + 1.0 / Z2p);
  c->eta_s = 1.0 / (1.0 / Z1s + 1.0 / Z2s);
  c->phi[0] = c->eta_p * (c->q[0] / Z2p - c->p[0] / Z1p);
  c->phi[1] = c->eta_s * (c->q[1] / Z2s - c->p[1] / Z1s);
  c->phi[2] = c->eta_s * (c->q[2] / Z2s - c->p[2] / Z1s);
}

/* Welded_Interface, src/Interface_Condition.f90:504-598 */
static void welded(const double *U, const double *V, double *P, double *Q, double Z1s, double Z2s, double Z1p,
                   double Z2p) {
  char_t c;
  characteristics(U, V, Z1s, Z2s, Z1p, Z2p, &c);
  P[0] = (c.q[0] - c.phi[0]) / Z2p; P[3] = c.phi[0];
  Q[0] = (c.p[0] + c.phi[0]) / Z1p; Q[3] = c.phi[0];
  P[2] = (c.q[2] - c.phi[2]) / Z2s; P[5] = c.phi[2];
  Q[2] = (c.p[2] + c.phi[2]) / Z1s; Q[5] = c.phi[2];
  P[1] = (c.q[1] - c.phi[1]) / Z2s; P[4] = c.phi[1];
  Q[1] = (c.p[1] + c.phi[1]) / Z1s; Q[4] = c.phi[1];
}

/* Linear_Friction, src/Interface_Condition.f90:601-741.  The reference never
   assigns u_out(2) (P_loc(2) keeps a stale value); this restatement sets it to
   the u_m_hat that the routine computes. */
static void linear_friction(const double *U, const double *V, double *P, double *Q, double Z1s, double Z2s,
                            double Z1p, double Z2p, double alpha) {
  char_t c;
  characteristics(U, V, Z1s, Z2s, Z1p, Z2p, &c);
  P[0] = (c.q[0] - c.phi[0]) / Z2p; P[3] = c.phi[0];
  Q[0] = (c.p[0] + c.phi[0]) / Z1p; Q[3] = c.phi[0];
  double tm = alpha / (alpha + c.eta_s) * c.phi[1];
  double tl = alpha / (alpha + c.eta_s) * c.phi[2];
  P[4] = tm; P[5] = tl; Q[4] = tm; Q[5] = tl;
  Q[1] = (c.p[1] + tm) / Z1s + 1.0 / (alpha + c.eta_s) * c.phi[1];
  Q[2] = (c.p[2] + tl) / Z1s + 1.0 / (alpha + c.eta_s) * c.phi[2];
  P[1] = (c.q[1] - tm) / Z2s - 1.0 / (alpha + c.eta_s) * c.phi[1];
  P[2] = (c.q[2] - tl) / Z2s - 1.0 / (alpha + c.eta_s) * c.phi[2];
}

/* Slip_Weakening_Friction with the closed-form solve,
   src/Interface_Condition.f90:745-916 and 1095-1168 */
static void slip_weakening(const oiface *I, long k, const double x[3], const double n[3], const double m[3],
                           const double l[3], const double *U, const double *V, double *P, double *Q, double Z1s,
                           double Z2s, double Z1p, double Z2p, double slip) {
  char_t c;
  characteristics(U, V, Z1s, Z2s, Z1p, Z2p, &c);
  double T0n, T0m, T0l;
  fault_prestress(I, k, x, n, m, l, &T0n, &T0m, &T0l);
  P[0] = (c.q[0] - c.phi[0]) / Z2p; P[3] = c.phi[0];
  Q[0] = (c.p[0] + c.phi[0]) / Z1p; Q[3] = c.phi[0];
  double tau_lock = sqrt((T0l + c.phi[2]) * (T0l + c.phi[2]) + (T0m + c.phi[1]) * (T0m + c.phi[1]));
  double sigma_n = fmax(0.0, -(T0n + c.phi[0]));
  double tau_str = fault_strength(I, k, x, sigma_n, slip);
  double tm_hat, tl_hat, vm, vl;
  if (tau_lock > tau_str) {
    double phi1 = T0m + c.phi[1], phi2 = T0l + c.phi[2];
    double Phi = sqrt(phi1 * phi1 + phi2 * phi2);
    double Vs = (Phi - tau_str) / c.eta_s;
    vm = phi1 / (c.eta_s + tau_str / Vs);
    vl = phi2 / (c.eta_s + tau_str / Vs);
    double tau_m = phi1 - c.eta_s * vm;
    double tau_l = phi2 - c.eta_s * vl;
    tm_hat = tau_m - T0m;
    tl_hat = tau_l - T0l;
  } else {
    tm_hat = c.phi[1];
    tl_hat = c.phi[2];
    vm = 0.0; vl = 0.0;
  }
  Q[1] = (tm_hat + c.p[1]) / Z1s + vm;
  Q[2] = (tl_hat + c.p[2]) / Z1s + vl;
  P[1] = (c.q[1] - tm_hat) / Z2s - vm;
  P[2] = (c.q[2] - tl_hat) / Z2s - vl;
  P[4] = tm_hat; P[5] = tl_hat; Q[4] = tm_hat; Q[5] = tl_hat;
}

/* smooth_boxcar, src/Interface_Condition.f90:2460-2476 */
static double smooth_boxcar(double x, double w, double wr) {
  if (-w <= x && x <= w) return 1.0;
  if (fabs(x) > w && fabs(x) < w + wr) return 0.5 * (1.0 + tanh(wr / (fabs(x) - w - wr) + wr / (fabs(x) - w)));
  return 0.0;
}

/* TPV101 / TPV102 rate-and-state parameters, src/Interface_Condition.f90:386-401 */
#define RS_L0 0.02
#define RS_F0 0.6
#define RS_B 0.012
#define RS_V0 1.0e-6
static double rs_a(const double x[3]) {
  return 0.008 + 0.008 * (1.0 - smooth_boxcar(x[1], 15.0, 3.0) * smooth_boxcar(x[2], 15.0, 3.0));
}

/* TPV101 / TPV102 prestress in the face basis at time t: the initial stress of
   src/initial_stress_condition.f90:114-120 as tractions on n, rotated onto
   n, m, l, plus the nucleation ramp 25 F(r) G(t) on T0_l
   (src/Interface_Condition.f90:2324-2385) */
static void rs_prestress(const double x[3], double t, const double n[3], const double m[3], const double l[3],
                         double *T0n, double *T0m, double *T0l) {
  const double sxx = -120.0, syy = 0.0, szz = -120.0, sxy = 0.0, sxz = 75.0, syz = 0.0;
  double Tx = n[0] * sxx + n[1] * sxy + n[2] * sxz;
  double Ty = n[0] * sxy + n[1] * syy + n[2] * syz;
  double Tz = n[0] * sxz + n[1] * syz + n[2] * szz;
  *T0n = n[0] * Tx + n[1] * Ty + n[2] * Tz;
  *T0m = m[0] * Tx + m[1] * Ty + m[2] * Tz;
  *T0l = l[0] * Tx + l[1] * Ty + l[2] * Tz;
  double r = sqrt((x[1] - 7.5) * (x[1] - 7.5) + x[2] * x[2]);
  double F = 0.0;
  if (r < 3.0) F = exp(r * r / (r * r - 9.0));
  double G = 0.0;
  if (t > 0.0 && t < 1.0) G = exp((t - 1.0) * (t - 1.0) / (t * (t - 2.0)));
  if (t >= 1.0) G = 1.0;
  *T0l = *T0l + 25.0 * F * G;
}

/* f(V) = V + a sigma_n / eta asinh(V / (2 V0) exp(psi / a)) - Phi / eta,
   src/Interface_Condition.f90:1242-1263 */
static double rs_f(double V, double Phi, double eta, double sn, double psi, double a) {
  return V + a * sn / eta * asinh(0.5 * V / RS_V0 * exp(psi / a)) - Phi / eta;
}

/* Regula_Falsi, src/Interface_Condition.f90:1170-1239: bracket [0, Phi/eta],
   absolute tolerance 1e-12, at most 5000 iterations */
static double rs_regula_falsi(double V, double Phi, double eta, double sn, double psi, double a) {
  const double tol = 1.0e-12;
  double Vl = 0.0, Vr = Phi / eta;
  double fv = rs_f(V, Phi, eta, sn, psi, a);
  double fl = rs_f(Vl, Phi, eta, sn, psi, a);
  double fr = rs_f(Vr, Phi, eta, sn, psi, a);
  if (fabs(fv) <= tol) return V;
  if (fabs(fl) <= tol) return Vl;
  if (fabs(fr) <= tol) return Vr;
  double err = 1.0;
  for (int k = 1; k <= 5000 && err >= tol; ++k) {
    double V1 = V;
    if (fv * fl > tol) {
      Vl = V;
      V = Vr - (Vr - Vl) * fr / (fr - fl);
      fl = fv;
    } else if (fv * fr > tol) {
      Vr = V;
      V = Vr - (Vr - Vl) * fr / (fr - fl);
      fr = fv;
    }
    fv = rs_f(V, Phi, eta, sn, psi, a);
    err = fabs(V - V1);
  }
  return V;
}

/* rate_state_friction + solve('rate-and-state_friction'),
   src/Interface_Condition.f90:918-1067, 1095-1168; *Vrs: the solved slip rate */
static void rate_state(const double x[3], double t, const double n[3], const double m[3], const double l[3],
                       const double *U, const double *V, double *P, double *Q, double Z1s, double Z2s, double Z1p,
                       double Z2p, double psi, double *Vrs) {
  char_t c;
  characteristics(U, V, Z1s, Z2s, Z1p, Z2p, &c);
  double T0n, T0m, T0l;
  rs_prestress(x, t, n, m, l, &T0n, &T0m, &T0l);
  P[0] = (c.q[0] - c.phi[0]) / Z2p; P[3] = c.phi[0];
  Q[0] = (c.p[0] + c.phi[0]) / Z1p; Q[3] = c.phi[0];
  double sigma_n = fmax(0.0, -(T0n + c.phi[0]));
  double a = rs_a(x);
  double vm = V[1] - U[1], vl = V[2] - U[2];
  double phi1 = T0m + c.phi[1], phi2 = T0l + c.phi[2];
  double Phi = sqrt(phi1 * phi1 + phi2 * phi2);
  double Vs = sqrt(vm * vm + vl * vl);
  if (Vs > Phi) Vs = 0.5 * Phi / c.eta_s;
  Vs = rs_regula_falsi(Vs, Phi, c.eta_s, sigma_n, psi, a);
  double fv = sigma_n * a * asinh(0.5 * Vs / RS_V0 * exp(psi / a));
  vm = phi1 / (c.eta_s + fv / Vs);
  vl = phi2 / (c.eta_s + fv / Vs);
  double tm = (phi1 - c.eta_s * vm) - T0m;
  double tl = (phi2 - c.eta_s * vl) - T0l;
  Q[1] = (tm + c.p[1]) / Z1s + vm;
  Q[2] = (tl + c.p[2]) / Z1s + vl;
  P[1] = (c.q[1] - tm) / Z2s - vm;
  P[2] = (c.q[2] - tl) / Z2s - vl;
  P[4] = tm; P[5] = tl; Q[4] = tm; Q[5] = tl;
  *Vrs = Vs;
}

/* init_vel_state for TPV101 / TPV102 as the one-process run calls it
   (src/domain.f90:273, src/Interface_Condition.f90:2722-2786): block 1's v_z
   set to -Vin/2 (Vin = 1e-12), and the state W from block 1's q-max face
   traction at t = 0: theta = L0/V0 exp((a log(2 sinh(T0_l/(a sigma_n))) - f0
   - a log(Vin/V0))/b), W = f0 + b log(V0/L0 theta).  V0 there is an
   unsuffixed literal: single precision unless the reals are promoted, so it
   follows the block's closure-literal switch. */
static void rs_init_vel_state(odom *D) {
  oblk *b = D->B[0];
  oiface *I = D->I;
  const double Vin = 1.0e-12;
  for (int z = 1; z <= b->nz; ++z)
    for (int y = 1; y <= b->ny; ++y)
      for (int x = 1; x <= b->nx; ++x) b->F[2][ID(b, x, y, z)] = -(0.5 * Vin);
  const double V0 = b->d.f32lit ? (double)1.0e-6f : 1.0e-6;
  for (int z = 1; z <= b->nz; ++z)
    for (int y = 1; y <= b->ny; ++y) {
      long k = (long)(y - 1) + (long)b->ny * (z - 1);
      long p = ID(b, b->nx, y, z);
      double x[3] = {b->X[0][p], b->X[1][p], b->X[2][p]};
      double n[3], m[3], l[3];
      for (int c = 0; c < 3; ++c) { n[c] = b->nn[1][c][k]; m[c] = b->nm[1][c][k]; l[c] = b->nl[1][c][k]; }
      double T0n, T0m, T0l;
      rs_prestress(x, 0.0, n, m, l, &T0n, &T0m, &T0l);
      double a = rs_a(x);
      double sigma_n = -T0n;
      double theta = RS_L0 / V0 * exp(((a * log(2.0 * sinh(T0l / (a * sigma_n)))) - RS_F0 - a * log(Vin / V0)) / RS_B);
      I->W[k] = RS_F0 + RS_B * log(V0 / RS_L0 * theta);
    }
}

static void rotate_in(double *w, const double n[3], const double m[3], const double l[3]) {
  /* src/CouplingForcing.f90:466-520 */
  double a[6];
  memcpy(a, w, sizeof a);
  w[0] = n[0] * a[0] + n[1] * a[1] + n[2] * a[2];
  w[1] = m[0] * a[0] + m[1] * a[1] + m[2] * a[2];
  w[2] = l[0] * a[0] + l[1] * a[1] + l[2] * a[2];
  w[3] = n[0] * a[3] + n[1] * a[4] + n[2] * a[5];
  w[4] = m[0] * a[3] + m[1] * a[4] + m[2] * a[5];
  w[5] = l[0] * a[3] + l[1] * a[4] + l[2] * a[5];
}

static void rotate_back(double *w, const double n[3], const double m[3], const double l[3]) {
  /* src/CouplingForcing.f90:524-580 */
  double a[6];
  memcpy(a, w, sizeof a);
  for (int i = 0; i < 3; ++i) {
    w[i] = n[i] * a[0] + m[i] * a[1] + l[i] * a[2];
    w[3 + i] = n[i] * a[3] + m[i] * a[4] + l[i] * a[5];
  }
}

/* SAT vector of one side from grid (g) and hat (h) values in x,y,z components:
   src/CouplingForcing.f90:250-437.  side 1: characteristics p = 1/2 (Zu + T)
   with the block-1 impedances, side 2: q = 1/2 (Zv - T) with block 2's, signs
   flipped on the stress rows. */
static void iface_sat(int side, const double *g, const double *h, double lambda, double mu, double rho,
                      const double n[3], const double m[3], const double l[3], double qx, double qy, double qz,
                      double *out) {
  double c_p = sqrt((2.0 * mu + lambda) / rho), c_s = sqrt(mu / rho);
  double Zp = rho * c_p, Zs = rho * c_s;
  double norm = sqrt(qx * qx + qy * qy + qz * qz);
  const double *e[3] = {n, m, l};
  double Mz[3][3], Mi[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      Mz[i][j] = e[i][0] * e[j][0] * Zp + e[i][1] * e[j][1] * Zs + e[i][2] * e[j][2] * Zs;
      Mi[i][j] = e[i][0] * e[j][0] * 1.0 / Zp + e[i][1] * e[j][1] * 1.0 / Zs + e[i][2] * e[j][2] * 1.0 / Zs;
    }
  double sg = side == 1 ? 1.0 : -1.0;
  double dch[3];
  for (int i = 0; i < 3; ++i) {
    double chat = 0.5 * (Mz[i][0] * h[0] + Mz[i][1] * h[1] + Mz[i][2] * h[2] + sg * h[3 + i]);
    double cg = 0.5 * (Mz[i][0] * g[0] + Mz[i][1] * g[1] + Mz[i][2] * g[2] + sg * g[3 + i]);
    dch[i] = cg - chat;
  }
  double r[3];
  for (int i = 0; i < 3; ++i) r[i] = Mi[i][0] * dch[0] + Mi[i][1] * dch[1] + Mi[i][2] * dch[2];
  double l2m = 2.0 * mu + lambda;
  for (int i = 0; i < 3; ++i) out[i] = norm / rho * dch[i];
  if (side == 1) {
    out[3] = l2m * qx * r[0] + lambda * qy * r[1] + lambda * qz * r[2];
    out[4] = l2m * qy * r[1] + lambda * qz * r[2] + lambda * qx * r[0];
    out[5] = l2m * qz * r[2] + lambda * qy * r[1] + lambda * qx * r[0];
    out[6] = mu * (qy * r[0] + qx * r[1]);
    out[7] = mu * (qz * r[0] + qx * r[2]);
    out[8] = mu * (qz * r[1] + qy * r[2]);
  } else {
    out[3] = -l2m * qx * r[0] - lambda * qy * r[1] - lambda * qz * r[2];
    out[4] = -l2m * qy * r[1] - lambda * qz * r[2] - lambda * qx * r[0];
    out[5] = -l2m * qz * r[2] - lambda * qy * r[1] - lambda * qx * r[0];
    out[6] = -mu * (qy * r[0] + qx * r[1]);
    out[7] = -mu * (qz * r[0] + qx * r[2]);
    out[8] = -mu * (qz * r[1] + qy * r[2]);
  }
}

/* Impose_Interface_Condition (src/RHS_Interior.f90:1771-1843) for block ib's
   side of the interface: ib == 2 is block 1 (its q-max face), ib == 1 is
   block 2 (its q-min face).  Couple_Interface_x (src/CouplingForcing.f90:9-463)
   builds tractions, rotates to (n, m, l), solves the interface law
   (Interface_RHS, src/Interface_Condition.f90:12-489), records the stage-1
   fault outputs, rotates back and forms the SAT vector of the calling side. */
void orc_iface_couple(odom *D, int ib, double t, int stage) {
  oiface *I = D->I;
  oblk *b = ib == 2 ? D->B[0] : D->B[1];
  int face = ib == 2 ? 1 : 0;            /* face index of the calling block */
  int xend = ib == 2 ? b->nx : 1;
  double *const *uF = ib == 2 ? b->faceF[1] : b->faceFopp[0];
  double *const *vF = ib == 2 ? b->faceFopp[1] : b->faceF[0];
  double *const *M1 = ib == 2 ? b->faceM[1] : b->faceMopp[0];
  double *const *M2 = ib == 2 ? b->faceMopp[1] : b->faceM[0];
  int accumulate = I->d.double_ds || ib == 2;
  int record = I->d.double_ds || ib == 2;
  const double pen = b->d.tau0 / b->hq;
  for (int z = 1; z <= b->nz; ++z)
    for (int y = 1; y <= b->ny; ++y) {
      long k = (long)(y - 1) + (long)b->ny * (z - 1);
      long p = ID(b, xend, y, z);
      double n[3], m[3], l[3];
      for (int c = 0; c < 3; ++c) { n[c] = b->nn[face][c][k]; m[c] = b->nm[face][c][k]; l[c] = b->nl[face][c][k]; }
      double u[6], v[6];
      u[0] = uF[0][k]; u[1] = uF[1][k]; u[2] = uF[2][k];
      u[3] = n[0] * uF[3][k] + n[1] * uF[6][k] + n[2] * uF[7][k];
      u[4] = n[0] * uF[6][k] + n[1] * uF[4][k] + n[2] * uF[8][k];
      u[5] = n[0] * uF[7][k] + n[1] * uF[8][k] + n[2] * uF[5][k];
      v[0] = vF[0][k]; v[1] = vF[1][k]; v[2] = vF[2][k];
      v[3] = n[0] * vF[3][k] + n[1] * vF[6][k] + n[2] * vF[7][k];
      v[4] = n[0] * vF[6][k] + n[1] * vF[4][k] + n[2] * vF[8][k];
      v[5] = n[0] * vF[7][k] + n[1] * vF[8][k] + n[2] * vF[5][k];
      rotate_in(u, n, m, l);
      rotate_in(v, n, m, l);
      /* Interface_RHS for this point */
      double lambda1 = M1[0][k], mu1 = M1[1][k], rho1 = M1[2][k];
      double lambda2 = M2[0][k], mu2 = M2[1][k], rho2 = M2[2][k];
      double c1p = sqrt((2.0 * mu1 + lambda1) / rho1), c1s = sqrt(mu1 / rho1);
      double c2p = sqrt((2.0 * mu2 + lambda2) / rho2), c2s = sqrt(mu2 / rho2);
      double Z1s = rho1 * c1s, Z2s = rho2 * c2s, Z1p = rho1 * c1p, Z2p = rho2 * c2p;
      double x[3] = {b->X[0][p], b->X[1][p], b->X[2][p]};
      double P[6], Q[6];
      double Vrs = 0.0;
      switch (I->d.coupling) {
        case ORC_IFACE_RATE_STATE:
          rate_state(x, t, n, m, l, u, v, P, Q, Z1s, Z2s, Z1p, Z2p, I->W[k], &Vrs);
          break;
        case ORC_IFACE_SLIP_WEAKENING:
          slip_weakening(I, k, x, n, m, l, u, v, P, Q, Z1s, Z2s, Z1p, Z2p, I->S[3][k]);
          break;
        case ORC_IFACE_LINEAR:
          linear_friction(u, v, P, Q, Z1s, Z2s, Z1p, Z2p, 1.0e14);
          break;
        default:
          welded(u, v, P, Q, Z1s, Z2s, Z1p, Z2p);
          break;
      }
      double Vel = sqrt((Q[1] - P[1]) * (Q[1] - P[1]) + (Q[2] - P[2]) * (Q[2] - P[2]));
      if (accumulate) {
        for (int c = 0; c < 3; ++c) I->DS[c][k] = I->DS[c][k] + Q[c] - P[c];
        I->DS[3][k] = I->DS[3][k] + Vel;
        /* rate of state, TPV101 / TPV102 (src/Interface_Condition.f90:431-436) */
        if (I->d.coupling == ORC_IFACE_RATE_STATE)
          I->DW[k] = I->DW[k] + RS_B * RS_V0 / RS_L0 * exp(-(I->W[k] - RS_F0) / RS_B) - Vrs * RS_B / RS_L0;
      }
      if (stage == 1 && record) {
        double T0n = 0.0, T0m = 0.0, T0l = 0.0;
        if (I->d.coupling == ORC_IFACE_RATE_STATE) rs_prestress(x, t, n, m, l, &T0n, &T0m, &T0l);
        else if (I->d.coupling != ORC_IFACE_LOCKED) fault_prestress(I, k, x, n, m, l, &T0n, &T0m, &T0l);
        /* Couple_Interface_x overwrites components 1:3 with v_hat - u_hat */
        for (int c = 0; c < 3; ++c) {
          double sv = Q[c] - P[c];
          I->Uhat[c][k] = sv; I->Vhat[c][k] = sv; I->Svel[c][k] = sv;
        }
        I->Uhat[3][k] = P[3] + T0n; I->Vhat[3][k] = Q[3] + T0n;
        I->Uhat[4][k] = P[4] + T0m; I->Vhat[4][k] = Q[4] + T0m;
        I->Uhat[5][k] = P[5] + T0l; I->Vhat[5][k] = Q[5] + T0l;
        /* rupture_front, src/CouplingForcing.f90:583-600 */
        if (sqrt(I->Svel[1][k] * I->Svel[1][k] + I->Svel[2][k] * I->Svel[2][k]) > 1.0e-3)
          I->trup[k] = fmin(I->trup[k], t);
      }
      rotate_back(u, n, m, l);
      rotate_back(v, n, m, l);
      rotate_back(P, n, m, l);
      rotate_back(Q, n, m, l);
      /* metric of the calling block at its interface face, used for both sides */
      double qx = b->mx[0][p], qy = b->my[0][p], qz = b->mz[0][p];
      double sat[9];
      if (ib == 2) iface_sat(1, u, P, lambda1, mu1, rho1, n, m, l, qx, qy, qz, sat);
      else iface_sat(2, v, Q, lambda2, mu2, rho2, n, m, l, qx, qy, qz, sat);
      for (int c = 0; c < 9; ++c) b->DF[c][p] = b->DF[c][p] - pen * sat[c];
    }
}

int orc_get_fault(void *dv, int kind, double *out) {
  odom *D = (odom *)dv;
  if (!D || !D->I) return -1;
  oiface *I = D->I;
  long n = (long)I->nr * I->ns;
  double **src = NULL;
  int nc = 0;
  switch (kind) {
    case ORC_FO_S: src = I->S; nc = 4; break;
    case ORC_FO_SVEL: src = I->Svel; nc = 3; break;
    case ORC_FO_UHAT: src = I->Uhat; nc = 6; break;
    case ORC_FO_VHAT: src = I->Vhat; nc = 6; break;
    case ORC_FO_STATE: src = &I->W; nc = 1; break;
    case ORC_FO_TRUP: src = &I->trup; nc = 1; break;
    default: return -1;
  }
  for (int c = 0; c < nc; ++c) memcpy(out + c * n, src[c], sizeof(double) * (size_t)n);
  return nc;
}


/* ======================================================================== */
/* Discrete adjoint of the elastic right-hand side (test infrastructure).   */
/*                                                                          */
/* For the rates R-bar of one stage, orc_adjoint_rhs adds L^T R-bar to the  */
/* field adjoint and (dL/dp F)^T R-bar to the material gradient, where L is */
/* this file's set_rates + impose_boundary_condition for one elastic block  */
/* (rhs_interior, rhs_near_boundaries with jju6 / jju_up, face SATs; no     */
/* PML, memory variables, interface or sources) and F the block's current   */
/* fields.  Written as the scatter transpose of those loops: every          */
/* accumulation DF[f][p] += c * F[g][q] there becomes Fbar[g][q] +=         */
/* c * Rbar[f][p] here.  SAT material derivatives by complex step.          */
/* ======================================================================== */
#include <complex.h>

/* adjoint of the rate assembly shared by the interior and near-boundary
   paths: DU = [a1 (Ux3 + Uy6 + Uz7), ...; a2 Ux0 + a3 (Uy1 + Uz2), ...;
   a4 (Uy0 + Ux1), ...]; returns the adjoints of Ux, Uy, Uz and adds the
   material gradient (a1 = 1 / (rho J) or 1 / rho) */
static void rates_adjoint(const double R[9], double a1, double lam, double mu, double rho, const double Ux[9],
                          const double Uy[9], const double Uz[9], double Ubx[9], double Uby[9], double Ubz[9],
                          double *glam, double *gmu, double *grho) {
  const double a2 = 2.0 * mu + lam, a3 = lam, a4 = mu;
  for (int f = 0; f < 9; ++f) { Ubx[f] = 0.0; Uby[f] = 0.0; Ubz[f] = 0.0; }
  Ubx[3] += a1 * R[0]; Uby[6] += a1 * R[0]; Ubz[7] += a1 * R[0];
  Ubx[6] += a1 * R[1]; Uby[4] += a1 * R[1]; Ubz[8] += a1 * R[1];
  Ubx[7] += a1 * R[2]; Uby[8] += a1 * R[2]; Ubz[5] += a1 * R[2];
  Ubx[0] += a2 * R[3] + a3 * R[4] + a3 * R[5];
  Uby[1] += a3 * R[3] + a2 * R[4] + a3 * R[5];
  Ubz[2] += a3 * R[3] + a3 * R[4] + a2 * R[5];
  Uby[0] += a4 * R[6]; Ubx[1] += a4 * R[6];
  Ubz[0] += a4 * R[7]; Ubx[2] += a4 * R[7];
  Ubz[1] += a4 * R[8]; Uby[2] += a4 * R[8];
  const double vs = R[0] * (Ux[3] + Uy[6] + Uz[7]) + R[1] * (Ux[6] + Uy[4] + Uz[8]) + R[2] * (Ux[7] + Uy[8] + Uz[5]);
  const double tr = Ux[0] + Uy[1] + Uz[2];
  *grho += -a1 / rho * vs;
  *glam += (R[3] + R[4] + R[5]) * tr;
  *gmu += 2.0 * (R[3] * Ux[0] + R[4] * Uy[1] + R[5] * Uz[2]) + R[6] * (Uy[0] + Ux[1]) + R[7] * (Uz[0] + Ux[2]) +
          R[8] * (Uz[1] + Uy[2]);
}

/* scatter transpose of one near-boundary derivative (jju6 or jju_up) for
   metric row X: Ub = adjoint of Ju; adds to Fbar */
static void jju_adjoint(const oblk *b, int x, int y, int z, double *const X[3], const double Ub[9], double **Fbar) {
  const long p0 = ID(b, x, y, z);
  const int pos[3] = {x, y, z}, nn[3] = {b->nx, b->ny, b->nz};
  const double ih[3] = {1.0 / b->hq, 1.0 / b->hr, 1.0 / b->hs};
  int cnt, idx[UP_MAXT];
  double c[UP_MAXT];
  const upwind_op *op = upwind_of(b->d.fd);
  for (int a = 0; a < 3; ++a)
    for (int grp = 0; grp < 2; ++grp) { /* 0: velocities, 1: stresses */
      if (op) up_stencil(op, grp == 0, pos[a], nn[a], &cnt, idx, c);
      else sbp_stencil(pos[a], nn[a], &cnt, idx, c);
      for (int k = 0; k < cnt; ++k) {
        const int q3[3] = {a == 0 ? idx[k] : x, a == 1 ? idx[k] : y, a == 2 ? idx[k] : z};
        const long q = ID(b, q3[0], q3[1], q3[2]);
        if (grp == 0)
          for (int f = 0; f < 3; ++f) Fbar[f][q] += ih[a] * X[a][p0] * c[k] * Ub[f];
        else
          for (int f = 3; f < 9; ++f) Fbar[f][q] += ih[a] * c[k] * b->J[q] * X[a][q] * Ub[f];
      }
    }
}

/* the SAT term pen * structure(bc_point(u)) of one face point in complex
   arithmetic (material perturbed by a complex step) */
static void sat_point_c(int plus, const double u[9], double complex rho, double complex mu, double complex lam,
                        const double l[3], const double m[3], const double n[3], double norm, double r, double pen,
                        double complex out[9]) {
  const double complex c_p = csqrt((2.0 * mu + lam) / rho), c_s = csqrt(mu / rho);
  const double complex Zp = rho * c_p, Zs = rho * c_s;
  double T[3];
  T[0] = n[0] * u[3] + n[1] * u[6] + n[2] * u[7];
  T[1] = n[0] * u[6] + n[1] * u[4] + n[2] * u[8];
  T[2] = n[0] * u[7] + n[1] * u[8] + n[2] * u[5];
  const double vl = l[0] * u[0] + l[1] * u[1] + l[2] * u[2];
  const double vm = m[0] * u[0] + m[1] * u[1] + m[2] * u[2];
  const double vn = n[0] * u[0] + n[1] * u[1] + n[2] * u[2];
  const double Tl = l[0] * T[0] + l[1] * T[1] + l[2] * T[2];
  const double Tm = m[0] * T[0] + m[1] * T[1] + m[2] * T[2];
  const double Tn = n[0] * T[0] + n[1] * T[1] + n[2] * T[2];
  const double s = plus ? 1.0 : -1.0;
  const double complex pl = 0.5 * ((1.0 - r) * Zs * vl + s * (1.0 + r) * Tl);
  const double complex pm = 0.5 * ((1.0 - r) * Zs * vm + s * (1.0 + r) * Tm);
  const double complex pn = 0.5 * ((1.0 - r) * Zp * vn + s * (1.0 + r) * Tn);
  const double complex ql = 0.5 * ((1.0 - r) * vl + s * (1.0 + r) / Zs * Tl);
  const double complex qm = 0.5 * ((1.0 - r) * vm + s * (1.0 + r) / Zs * Tm);
  const double complex qn = 0.5 * ((1.0 - r) * vn + s * (1.0 + r) / Zp * Tn);
  double complex ub[9];
  for (int c = 0; c < 3; ++c) ub[c] = norm * (l[c] * pl + m[c] * pm + n[c] * pn);
  const double complex Fx = l[0] * ql + m[0] * qm + n[0] * qn;
  const double complex Fy = l[1] * ql + m[1] * qm + n[1] * qn;
  const double complex Fz = l[2] * ql + m[2] * qm + n[2] * qn;
  ub[3] = s * (norm * n[0] * Fx);
  ub[4] = s * (norm * n[1] * Fy);
  ub[5] = s * (norm * n[2] * Fz);
  ub[6] = s * (norm * (n[1] * Fx + n[0] * Fy));
  ub[7] = s * (norm * (n[2] * Fx + n[0] * Fz));
  ub[8] = s * (norm * (n[2] * Fy + n[1] * Fz));
  out[0] = pen / rho * ub[0];
  out[1] = pen / rho * ub[1];
  out[2] = pen / rho * ub[2];
  out[3] = pen * ((2.0 * mu + lam) * ub[3] + lam * (ub[4] + ub[5]));
  out[4] = pen * ((2.0 * mu + lam) * ub[4] + lam * (ub[3] + ub[5]));
  out[5] = pen * ((2.0 * mu + lam) * ub[5] + lam * (ub[3] + ub[4]));
  out[6] = pen * (mu * ub[6]);
  out[7] = pen * (mu * ub[7]);
  out[8] = pen * (mu * ub[8]);
}

int orc_adjoint_rhs(void *dv, int bi, const double *Rin, double *Fbout, double *gout) {
  odom *D = (odom *)dv;
  oblk *b = D->B[bi];
  if (b->d.response != ORC_ELASTIC || b->d.mms) return -1;
  for (int f = 0; f < 6; ++f)
    if (b->d.pml[f] || b->d.bc[f] == 0) return -1;
  const long np = b->np;
  double *R[9], *Fb[9], *g[3];
  for (int f = 0; f < 9; ++f) { R[f] = zalloc(np, 0.0); Fb[f] = zalloc(np, 0.0); }
  for (int f = 0; f < 3; ++f) g[f] = zalloc(np, 0.0);
  set3(b, R, 9, Rin);
  int lo[3], hi[3];
  interior_bounds(b, lo, hi);
  const int curv = b->d.mesh == 1;
  const long st[3] = {1, b->NX, (long)b->NX * b->NY};
  for (int z = 1; z <= b->nz; ++z)
    for (int y = 1; y <= b->ny; ++y)
      for (int x = 1; x <= b->nx; ++x) {
        const long p = ID(b, x, y, z);
        double Rp[9];
        for (int f = 0; f < 9; ++f) Rp[f] = R[f][p];
        const double lam = b->M[0][p], mu = b->M[1][p], rho = b->M[2][p];
        const int interior = lo[2] <= z && z <= hi[2] && lo[1] <= y && y <= hi[1] && lo[0] <= x && x <= hi[0];
        double Ux[9] = {0}, Uy[9] = {0}, Uz[9] = {0}, Ubx[9], Uby[9], Ubz[9];
        if (!interior) {
          if (upwind_of(b->d.fd)) {
            const upwind_op *op = upwind_of(b->d.fd);
            jju_up(b, op, x, y, z, b->mx, Ux); jju_up(b, op, x, y, z, b->my, Uy); jju_up(b, op, x, y, z, b->mz, Uz);
          } else {
            jju6(b, x, y, z, b->mx, Ux); jju6(b, x, y, z, b->my, Uy); jju6(b, x, y, z, b->mz, Uz);
          }
          rates_adjoint(Rp, 1.0 / (rho * b->J[p]), lam, mu, rho, Ux, Uy, Uz, Ubx, Uby, Ubz, &g[0][p], &g[1][p],
                        &g[2][p]);
          jju_adjoint(b, x, y, z, b->mx, Ubx, Fb);
          jju_adjoint(b, x, y, z, b->my, Uby, Fb);
          jju_adjoint(b, x, y, z, b->mz, Ubz, Fb);
          continue;
        }
        /* strict interior: the forward's DFx / DFy / DFz as plain sums of tap terms */
        double ws[2][10];  /* per tap: coefficient / h */
        int offs[2][10], ntap[2];
        if (upwind_of(b->d.fd)) {
          const upwind_op *op = upwind_of(b->d.fd);
          ntap[0] = ntap[1] = op->taps;
          for (int k = 0; k < op->taps; ++k) {
            ws[0][k] = op->inf_[k]; offs[0][k] = op->of + k; ws[1][k] = op->inb[k]; offs[1][k] = op->ob + k;
          }
        } else {
          static const double cc[6] = {-1.0 / 60.0, 0.15, -0.75, 0.75, -0.15, 1.0 / 60.0};
          static const int oo[6] = {-3, -2, -1, 1, 2, 3};
          ntap[0] = ntap[1] = 6;
          for (int k = 0; k < 6; ++k) { ws[0][k] = ws[1][k] = cc[k]; offs[0][k] = offs[1][k] = oo[k]; }
        }
        const double ih[3] = {1.0 / b->hq, 1.0 / b->hr, 1.0 / b->hs};
        double *const *Xr[3] = {b->mx, b->my, b->mz};
        double DF3[3][9];  /* [row r] derivative terms DFx, DFy, DFz */
        for (int r = 0; r < 3; ++r)
          for (int f = 0; f < 9; ++f) DF3[r][f] = 0.0;
        for (int r = 0; r < 3; ++r)
          for (int a = 0; a < 3; ++a) {
            if (!curv && a != r) continue;
            for (int grp = 0; grp < 2; ++grp)
              for (int k = 0; k < ntap[grp]; ++k) {
                const long q = p + offs[grp][k] * st[a];
                for (int f = grp ? 3 : 0; f < (grp ? 9 : 3); ++f) {
                  const double w = ws[grp][k] * ih[a];
                  DF3[r][f] += (curv && grp) ? w * b->F[f][q] * b->J[q] * Xr[r][a][q] : Xr[r][a][p] * w * b->F[f][q];
                }
              }
          }
        const double a1 = curv ? 1.0 / (rho * b->J[p]) : 1.0 / rho;
        rates_adjoint(Rp, a1, lam, mu, rho, DF3[0], DF3[1], DF3[2], Ubx, Uby, Ubz, &g[0][p], &g[1][p], &g[2][p]);
        const double *Ub[3] = {Ubx, Uby, Ubz};
        for (int r = 0; r < 3; ++r)
          for (int a = 0; a < 3; ++a) {
            if (!curv && a != r) continue;
            for (int grp = 0; grp < 2; ++grp)
              for (int k = 0; k < ntap[grp]; ++k) {
                const long q = p + offs[grp][k] * st[a];
                const double w = ws[grp][k] * ih[a];
                for (int f = grp ? 3 : 0; f < (grp ? 9 : 3); ++f)
                  Fb[f][q] += ((curv && grp) ? w * b->J[q] * Xr[r][a][q] : Xr[r][a][p] * w) * Ub[r][f];
              }
          }
      }
  /* face SATs: DF(p) -= pen * structure(bc_point(u(p))), linear in u(p) */
  const double hs_[3] = {b->hq, b->hr, b->hs};
  for (int f = 0; f < 6; ++f) {
    const int type = b->d.bc[f];
    if (type <= 0) continue;
    const int axis = f / 2, plus = f % 2;
    const double r = type == 1 ? 0.0 : type == 2 ? 1.0 : -1.0;
    const int fixed = plus ? (axis == 0 ? b->nx : axis == 1 ? b->ny : b->nz) : 1;
    const double pen = b->d.tau0 / hs_[axis];
    for (int c2 = 1; c2 <= b->fdim[f][1]; ++c2)
      for (int c1 = 1; c1 <= b->fdim[f][0]; ++c1) {
        int x, y, z;
        if (axis == 0) { x = fixed; y = c1; z = c2; }
        else if (axis == 1) { x = c1; y = fixed; z = c2; }
        else { x = c1; y = c2; z = fixed; }
        const long p = ID(b, x, y, z);
        const long fp = FID(b, f, c1, c2);
        double l3[3], m3[3], n3[3], u[9];
        for (int c = 0; c < 3; ++c) { l3[c] = b->nl[f][c][fp]; m3[c] = b->nm[f][c][fp]; n3[c] = b->nn[f][c][fp]; }
        const double qx = b->mx[axis][p], qy = b->my[axis][p], qz = b->mz[axis][p];
        const double norm = sqrt(qx * qx + qy * qy + qz * qz);
        const double lam = b->M[0][p], mu = b->M[1][p], rho = b->M[2][p];
        double complex out[9];
        for (int j = 0; j < 9; ++j) { /* Jacobian column j (the term is linear in u) */
          for (int c = 0; c < 9; ++c) u[c] = c == j ? 1.0 : 0.0;
          sat_point_c(plus, u, rho, mu, lam, l3, m3, n3, norm, r, pen, out);
          double acc = 0.0;
          for (int c = 0; c < 9; ++c) acc += creal(out[c]) * R[c][p];
          Fb[j][p] -= acc;
        }
        const double hstep = 1e-30;
        for (int c = 0; c < 9; ++c) u[c] = b->F[c][p];
        for (int prm = 0; prm < 3; ++prm) { /* lambda, mu, rho */
          double complex cl = lam, cm = mu, cr = rho;
          if (prm == 0) cl += I * hstep;
          if (prm == 1) cm += I * hstep;
          if (prm == 2) cr += I * hstep;
          sat_point_c(plus, u, cr, cm, cl, l3, m3, n3, norm, r, pen, out);
          double acc = 0.0;
          for (int c = 0; c < 9; ++c) acc += cimag(out[c]) / hstep * R[c][p];
          g[prm][p] -= acc;
        }
      }
  }
  double *outF = Fbout, *outG = gout;
  double *tmp9 = (double *)malloc(sizeof(double) * 9 * (size_t)b->nx * b->ny * b->nz);
  get3(b, Fb, 9, tmp9);
  const long n = (long)b->nx * b->ny * b->nz;
  for (long i = 0; i < 9 * n; ++i) outF[i] += tmp9[i];
  get3(b, g, 3, tmp9);
  for (long i = 0; i < 3 * n; ++i) outG[i] += tmp9[i];
  free(tmp9);
  for (int f = 0; f < 9; ++f) { free(R[f]); free(Fb[f]); }
  for (int f = 0; f < 3; ++f) free(g[f]);
  return 0;
}

/* moment-tensor adjoint of the sources at time t: gM[6 * i + c] +=
   -A_i(t) sum_p delta_i(p) Rbar_(3+c)(p) (set_moment_tensor above) */
void orc_adjoint_moment(void *dv, int bi, double t, const double *Rin, double *gM) {
  odom *D = (odom *)dv;
  oblk *b = D->B[bi];
  const orc_desc *d = &b->d;
  const int half = d->src_order == 4 ? 4 : 2;
  const long n = (long)b->nx * b->ny * b->nz;
  for (int i = 0; i < b->nsrc; ++i) {
    const double *sp = &b->spar[i * 11];
    const int nx0 = b->snear[3 * i], ny0 = b->snear[3 * i + 1], nz0 = b->snear[3 * i + 2];
    if (nx0 < 1) continue;
    const double A = source_time(b->stype[i], t, sp[1], sp[0]);
    for (int k = nz0 - half; k <= nz0 + half; ++k) {
      if (k < 1 || k > b->nz) continue;
      for (int m = ny0 - half; m <= ny0 + half; ++m) {
        if (m < 1 || m > b->ny) continue;
        for (int l = nx0 - half; l <= nx0 + half; ++l) {
          if (l < 1 || l > b->nx) continue;
          const long p = ID(b, l, m, k);
          const double hx = b->hq / b->mx[0][p], hy = b->hr / b->my[1][p], hz = b->hs / b->mz[2][p];
          const double ax = (sp[8] - b->sphys[3 * i]) / hx, ay = (sp[9] - b->sphys[3 * i + 1]) / hy;
          const double az = (sp[10] - b->sphys[3 * i + 2]) / hz;
          const double delta = singular_source(l, nx0, hx, ax, d->src_order, d->src_alpha) *
                               singular_source(m, ny0, hy, ay, d->src_order, d->src_alpha) *
                               singular_source(k, nz0, hz, az, d->src_order, d->src_alpha);
          const long li = (long)(l - 1) + (long)b->nx * ((long)(m - 1) + (long)b->ny * (long)(k - 1));
          for (int c = 0; c < 6; ++c) gM[6 * i + c] -= A * delta * Rin[(3 + c) * n + li];
        }
      }
    }
  }
}

/* ======================================================================== */
/* Transfinite interpolation of a block from its six boundary surfaces,      */
/* Gen3_Curve_Mesh of src/grid.f90:2292-2418.  faces: left, right (3 x ns x  */
/* nr), top, bottom (3 x ns x nq), front, back (3 x nr x nq), first index    */
/* slowest; out: 3 x ns x nr x nq, q fastest.                                */
/* ======================================================================== */
void orc_tfi_grid(const double *faces, int nq, int nr, int ns, double *out) {
  const long nLR = 3L * ns * nr, nTB = 3L * ns * nq;
  const double *Lf = faces, *Rf = Lf + nLR, *Tf = Rf + nLR, *Bf = Tf + nTB, *Ff = Bf + nTB, *Kf = Ff + 3L * nr * nq;
  const double hq = 1.0 / (double)(nq - 1), hr = 1.0 / (double)(nr - 1), hs = 1.0 / (double)(ns - 1);
  const long npt = (long)nq * nr * ns;
#define TL(c, j, k) Lf[((long)(c) * ns + (k)) * nr + (j)]
#define TR(c, j, k) Rf[((long)(c) * ns + (k)) * nr + (j)]
#define TT(c, i, k) Tf[((long)(c) * ns + (k)) * nq + (i)]
#define TB(c, i, k) Bf[((long)(c) * ns + (k)) * nq + (i)]
#define TF(c, i, j) Ff[((long)(c) * nr + (j)) * nq + (i)]
#define TK(c, i, j) Kf[((long)(c) * nr + (j)) * nq + (i)]
  for (int c = 0; c < 3; ++c)
    for (int k = 0; k < ns; ++k)
      for (int j = 0; j < nr; ++j)
        for (int i = 0; i < nq; ++i) {
          const double q = (double)i * hq, r = (double)j * hr, s = (double)k * hs;
          const double U = (1.0 - q) * TL(c, j, k) + q * TR(c, j, k);
          const double V = (1.0 - r) * TT(c, i, k) + r * TB(c, i, k);
          const double W = (1.0 - s) * TF(c, i, j) + s * TK(c, i, j);
          const double UW = (1.0 - q) * ((1.0 - r) * TL(c, 0, k) + r * TL(c, nr - 1, k)) +
                            q * ((1.0 - r) * TR(c, 0, k) + r * TR(c, nr - 1, k));
          const double UV = (1.0 - r) * ((1.0 - s) * TT(c, i, 0) + s * TT(c, i, ns - 1)) +
                            r * ((1.0 - s) * TB(c, i, 0) + s * TB(c, i, ns - 1));
          const double VW = (1.0 - s) * ((1.0 - q) * TF(c, 0, j) + q * TF(c, nq - 1, j)) +
                            s * ((1.0 - q) * TK(c, 0, j) + q * TK(c, nq - 1, j));
          const double UVW1 = (1.0 - q) * ((1.0 - r) * ((1.0 - s) * TT(c, 0, 0) + s * TT(c, 0, ns - 1)) +
                                           r * ((1.0 - s) * TB(c, 0, 0) + s * TB(c, 0, ns - 1)));
          const double UVW2 = q * ((1.0 - r) * ((1.0 - s) * TT(c, nq - 1, 0) + s * TT(c, nq - 1, ns - 1)) +
                                   r * ((1.0 - s) * TB(c, nq - 1, 0) + s * TB(c, nq - 1, ns - 1)));
          out[(long)c * npt + ((long)k * nr + j) * nq + i] = U + V + W - UV - UW - VW + UVW1 + UVW2;
        }
#undef TL
#undef TR
#undef TT
#undef TB
#undef TF
#undef TK
}
