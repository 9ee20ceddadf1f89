/* cpsb200.h -- C ABI of the B200 fermion-matrix library (libcpsb200.so).
 *
 * A drop-in device implementation of the CPS (RBC-UKQCD/CPS_public, cps_pp)
 * fermion-matrix hot path: the even-odd preconditioned Wilson, Shamir
 * domain-wall and Mobius operators and the CG / multishift-CG solvers that
 * drive them.  Every entry point replaces one CPS interface, cited below by
 * file:line relative to cps_pp/.  Vectors use CPS storage order: a checkerboard
 * vector is sites x 24 doubles (r + 2*(colour + 3*spin)); a 5-D vector is Ls
 * consecutive 4-D slices (5-D checkerboarding for DWF, the DWF_4D_EOPREC_EE
 * half for Mobius), exactly as DiracOp*::MatPcDagMatPc receives it.
 *
 * Errors are reported as status codes (CPS instead prints through ERR and
 * calls exit(), include/util/error.h:26-80): 0 ok, 1 not converged within
 * max_num_iter (CPS only warns, inv_cg.C:392-396), negative values are errors.
 * Host-pointer entry points copy in and out and keep no host pointer after
 * returning; gauge handles stay resident on the device until freed.
 */
#ifndef CPSB200_H
#define CPSB200_H

#ifdef __cplusplus
extern "C" {
#endif

#define CPSB_OK 0
#define CPSB_NOT_CONVERGED 1
#define CPSB_ERR_ARG (-1)
#define CPSB_ERR_CUDA (-2)
#define CPSB_ERR_OOM (-3)
#define CPSB_ERR_UNSUPPORTED (-4)
#define CPSB_ERR_BREAKDOWN (-5)
#define CPSB_ERR_NO_DEVICE (-6)
#define CPSB_ERR_BUSY (-7)

enum cpsb_action { CPSB_WILSON = 0, CPSB_DWF = 1, CPSB_MOBIUS = 2, CPSB_ZMOBIUS = 3 };
enum cpsb_precision { CPSB_PREC_F64 = 0, CPSB_PREC_F32 = 1, CPSB_PREC_F16 = 2 };
enum cpsb_gauge_order { CPSB_ORDER_CANONICAL = 0, CPSB_ORDER_WILSON = 1 };
enum cpsb_multishift_type { CPSB_MULTI = 0, CPSB_SINGLE = 1 };
enum cpsb_fermion_order { CPSB_FERMION_CB = 0, CPSB_FERMION_4D_EE = 1 };

typedef struct cpsb_gauge_s *cpsb_gauge;

/* Operator parameters: the fields CPS reads from CgArg and GJP.
 *   mass    CgArg::mass (include/alg/cg_arg.h:17-36).  Wilson: kappa =
 *           1/(2(mass+4)) (d_op_wilson/noarch/d_op_wilson.C:134-137); DWF and
 *           Mobius: the domain-wall mass m_f.
 *   m5      GJP.DwfHeight() (include/util/gjp.h:579)
 *   a5_inv  GJP.DwfA5Inv() (gjp.h:587)
 *   mobius_b, mobius_c   GJP.Mobius_b/c() (gjp.h:594-601)
 *   pc_type GJP.ZMobius_PC_Type() (include/util/dwf.h:42-48): ZMOB_PC_ORIG (0),
 *           ZMOB_PC_SYM1 (1) and ZMOB_PC_SYM2 (2, the CPS default, src/util/gjp/
 *           gjp.C:129) for Mobius; for zMobius also ZMOB_PC_SYM1_MIT (3),
 *           ZMOB_PC_SYM2_MIT (4) and ZMOB_PC_SYM3 (5).  Other values (and the MIT
 *           and SYM3 forms for real Mobius, where the reference reads empty
 *           zMobius coefficient arrays) return CPSB_ERR_UNSUPPORTED.
 *   zmobius_b, zmobius_c   zMobius (CPSB_ZMOBIUS) only: the complex per-slice
 *           coefficients b_s, c_s as ls (re, im) pairs each, the layout of
 *           DoArgExt::zmobius_b_coeff / zmobius_c_coeff (GJP.ZMobius_b/c(),
 *           src/util/gjp/gjp.C:167-178).  Read during the call only (solvers
 *           and the request loop keep copies); ignored for the other actions. */
typedef struct {
  int action;
  int ls;
  double mass;
  double m5;
  double a5_inv;
  double mobius_b;
  double mobius_c;
  int pc_type;
  const double *zmobius_b;
  const double *zmobius_c;
} cpsb_dirac_params;

/* Solver controls: CgArg::stop_rsd / max_num_iter plus the precision forms.
 *   precision       inner (sloppy) precision; CPSB_PREC_F64 runs the plain CPS
 *                   CG recurrence in FP64
 *   reliable_delta  FP64 residual replacement whenever |r| drops by this factor
 *                   since the last one (mixed precision only; 0 -> 0.1)
 *   batch           iterations launched per device batch (0 -> automatic) */
typedef struct {
  double stop_rsd;
  int max_num_iter;
  int precision;
  double reliable_delta;
  int batch;
} cpsb_cg_arg;

/* Per-solve report.  iters follows CPS (DiracOp::InvCg returns itr+1,
 * inv_cg.C:444); true_rsd = |b - A x|/|b| computed in FP64 after the solve
 * (inv_cg.C:401-417). */
typedef struct {
  int iters;
  double true_rsd;
  double iter_rsd;
  int reliable_updates;
  double seconds;
  int status;
} cpsb_solve_result;

/* Selects the CUDA device and creates the library context (one per process):
 * the device half of CPS's Start(), which in QUDA builds calls
 * initQuda(QudaParam.device) (src/util/gjp/qmp/start_end.C:54). */
int cpsb_init(int device);
const char *cpsb_error_string(int code);
/* Detail message of the last error raised on the calling thread. */
const char *cpsb_last_error(void);
/* Free and total device memory in bytes (the serving loop admits work by it).
 * No counterpart in the reference. */
int cpsb_mem_info(unsigned long long *free_bytes, unsigned long long *total_bytes);

/* Uploads a gauge field and keeps it resident (FP64 plus the reduced-precision
 * copies made on first use).  u: 4*V 3x3 complex links; order CANONICAL
 * (Lattice::GaugeField(), lattice/convert/convert_func.C:397-405) or WILSON
 * (the order DiracOp constructors convert to, convert_func.C:371-405).
 * bc_t = 1 applies the antiperiodic time boundary as Lattice::BondCond does
 * (lattice/lattice_base/lattice_base.C:5313-5370).  Replaces the gauge half of
 * the DiracOp constructor (d_op_dwf/d_op_dwf.C:67-123). */
int cpsb_gauge_load(cpsb_gauge *h, const double *u, const int dims[4], int order, int bc_t);
/* Releases a resident field and the solvers built on it: the device end of the
 * DiracOp destructor's conversion back to CANONICAL (d_op_dwf/d_op_dwf.C:132-150)
 * and of freeGaugeQuda in the QUDA bridge (d_op_dwf/quda/dwf_quda.C:173).
 * Returns CPSB_ERR_BUSY (and frees nothing) while requests of the request loop
 * (cpsb_serve_submit*) on this field are queued or running: wait for them
 * first.  A solve running on another host thread is waited for.  The handle
 * must not be used by any call that starts after this one. */
int cpsb_gauge_free(cpsb_gauge h);

/* DiracOp*::Dslash(out, in, cb, dag) (include/util/dirac_op.h:275):
 * d_op_wilson/noarch/d_op_wilson.C:180 (wilson_dslash), d_op_dwf/d_op_dwf.C:210
 * (dwf_dslash), d_op_mobius/d_op_mobius.C:273 (mobius_dslash). */
int cpsb_dslash(cpsb_gauge h, const cpsb_dirac_params *p, double *out, const double *in, int cb, int dag);

/* DiracOp*::MatPc (dag = 0) / MatPcDag (dag = 1): d_op_wilson.C:204,228;
 * d_op_dwf.C:245-300; d_op_mobius.C:319-372. */
int cpsb_matpc(cpsb_gauge h, const cpsb_dirac_params *p, double *out, const double *in, int dag);

/* DiracOp*::MatPcDagMatPc(out, in, dot_prd) (dirac_op.h:262); dot, when not
 * NULL, receives |MatPc in|^2 as CPS's fused norm does (dwf_mdagm.C:49-55). */
int cpsb_mdagm(cpsb_gauge h, const cpsb_dirac_params *p, double *out, const double *in, double *dot);

/* DiracOp::InvCg through Lattice::FmatEvlInv(f_out, f_in, cg_arg, true_res)
 * (include/util/lattice.h:942; lattice/f_wilson/f_wilson.C:159,
 * f_dwf_base/f_dwf_base.C:189, f_mobius/f_mobius.C:582): solves
 * MatPcDagMatPc x = b by CG from the initial guess in x. */
int cpsb_invcg(cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a, double *x, const double *b,
               cpsb_solve_result *res);

/* nrhs independent solves batched into one launch sequence (each link load
 * serves all right-hand sides): the multi-source DiracOpMobius::MatInv
 * (dirac_op.h:1886) / QUDA split-grid path (d_op_mobius/noarch/mobius_quda.C:32-340)
 * at the FmatEvlInv level.  x[i], b[i]: nrhs host vectors; res: nrhs reports. */
int cpsb_invcg_multi(cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a, int nrhs, double **x,
                     const double *const *b, cpsb_solve_result *res);

/* DiracOp::MInvCG via Lattice::FmatEvlMInv (lattice.h:976; f_dwf_base.C:232,
 * f_mobius.C:628; d_op_base/noarch/minvcg.C:47-353): solves
 * (MatPcDagMatPc + shift[s]) x[s] = b for all shifts (shift[0] the smallest).
 * type CPSB_MULTI writes x[0..nshift); CPSB_SINGLE writes sum_s alpha[s] x_s to
 * x[0].  rsd[s]: stop_rsd per shift on entry; on return the residual reported
 * per shift.  With a->precision != F64 the Krylov vectors are kept in that
 * precision and every shift is then refined by mixed-precision CG to its
 * tolerance with an FP64 true residual (rsd[s] then holds that true residual).
 * CPS's third type, GENERAL (2, include/alg/enum_int.h:236: start from the
 * guess in x[0], minvcg.C:125-129), has no caller in CPS and returns
 * CPSB_ERR_UNSUPPORTED.  Its first solution update subtracts bs[s]*chi where
 * the recurrence needs bs[s]*r (minvcg.C:174-184).  Replayed on a small SPD
 * system with a nonzero guess, every shift ends at relative residual ~1, not the
 * tolerance.  With bs[s]*r, shift 0 converges, but the other shifts still stop
 * short: one guess breaks the collinearity of their residuals with r. */
int cpsb_minvcg(cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a, double **x, const double *b,
                const double *shift, int nshift, double *rsd, int type, const double *alpha,
                cpsb_solve_result *res);

/* DiracOp*::MatInv(out, in, true_res, PRESERVE_YES) (include/util/dirac_op.h:294)
 * and Lattice::FmatInv (lattice.h:1114): the full-lattice solve.  in, out are
 * full vectors of both checkerboards in the action's order (Wilson, DWF: odd
 * half first, d_op_wilson.C:284-287, d_op_dwf.C:316-507; Mobius: even half first,
 * d_op_mobius.C:389-640, ZMOB_PC_SYM2 only).  The solve-checkerboard half of out
 * is the CG's initial guess on entry.  Source preparation, MatPcDag, the CG (of
 * the requested precision) and the reconstruction of the other checkerboard run
 * on the device; res reports the CG as cpsb_invcg does. */
int cpsb_matinv(cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a, double *out, const double *in,
                cpsb_solve_result *res);

/* Lattice::FmatInv(f_out, f_in, cg_arg, true_res, CNV_FRM_NO, PRESERVE_YES, dminus)
 * (lattice.h:1127-1132; Fmobius override f_mobius.C:45-117): for Mobius with
 * dminus != 0 the source is first replaced by DiracOpMobius::Dminus of it (on the
 * device; in is not modified), then the solve is cpsb_matinv's.  Wilson and DWF
 * ignore dminus, as the reference's default FmatInv does. */
int cpsb_fmatinv(cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a, double *out, const double *in,
                 int dminus, cpsb_solve_result *res);

/* DiracOpMobius::Dminus(out, in) (d_op_mobius.C:745-777, mobius_dminus.C:29-86) on
 * full Mobius vectors (4-D-even half first): out = -(c(4 - M5) - a5_inv) in
 * + (c/2) D_W in, D_W the 4-D hop of every s slice into the other checkerboard.
 * zMobius: DiracOpZMobius::Dminus (d_op_zmobius.C:1213-1272) with the complex c_s
 * of each slice, on its full vectors (odd half first).  Mobius and zMobius only
 * (CPSB_ERR_ARG otherwise); out and in must not overlap. */
int cpsb_dminus(cpsb_gauge h, const cpsb_dirac_params *p, double *out, const double *in);

/* DiracOp::MinResExt(psi, phi, v, vm, degree) (include/util/dirac_op.h;
 * d_op_base/comsrc/minresext.C:32-156): the minimal-residual chronological
 * initial guess from degree <= 16 previous solutions.  v[i] (host vectors) are
 * orthonormalised in place, vm[i] receive MatPcDagMatPc v[i], psi the guess;
 * resid (optional) receives |phi - MatPcDagMatPc psi| / |phi|.  The vector
 * work runs on the device, the degree x degree elimination on the host. */
int cpsb_minresext(cpsb_gauge h, const cpsb_dirac_params *p, double *psi, const double *phi, double **v,
                   double **vm, int degree, double *resid);

/* Lattice::Fconvert for fermion fields (include/util/lattice.h:1326;
 * lattice/convert/convert_func.C:429-495, convert.C:635-1010) on the device:
 * CANONICAL (slice s slowest, then site x+lx*(y+ly*(z+lz*t))) <-> the
 * checkerboarded order the solvers take.  order CPSB_FERMION_CB: WILSON
 * (odd 4-D half first; for ls > 1 the 5-D checkerboard, sites with x+y+z+t+s
 * odd first); CPSB_FERMION_4D_EE: DWF_4D_EOPREC_EE (Mobius: 4-D even half of
 * every slice first).  direction 0: CANONICAL -> order, 1: order -> CANONICAL.
 * out, in: distinct device buffers of vol*ls*24 doubles. */
int cpsb_fermion_convert(const int dims[4], int ls, int order, int direction, double *out, const double *in,
                         void *stream);

/* Device-resident variants: x, b (and out/in) are device pointers holding CPS
 * order vectors; stream is a cudaStream_t (NULL = the library stream).  These
 * are what a caller with fields already in HBM uses. */
int cpsb_invcg_dev(cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a, double *x, const double *b,
                   cpsb_solve_result *res, void *stream);
int cpsb_invcg_multi_dev(cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a, int nrhs, double *x,
                         const double *b, cpsb_solve_result *res, void *stream);
int cpsb_mdagm_dev(cpsb_gauge h, const cpsb_dirac_params *p, double *out, const double *in, double *dot,
                   void *stream);
/* The multi-right-hand-side Dslash and MatPcDagMatPc: the operator applied to
 * nrhs vectors in one launch sequence, every link read once for all of them,
 * with fields stored in the given precision (as cpsb_dslash_ex).  in, out:
 * device pointers to nrhs consecutive CPS-order vectors; dot (host, nrhs
 * entries, may be NULL) receives |MatPc in_q|^2.  Interfaces of DiracOp::Dslash
 * (dirac_op.h:275) and DiracOp::MatPcDagMatPc (dirac_op.h:262), which CPS
 * applies one vector at a time (its multi-source DiracOpMobius::MatInv,
 * dirac_op.h:1886, loops over the sources). */
int cpsb_dslash_multi_dev(cpsb_gauge h, const cpsb_dirac_params *p, int precision, int nrhs, double *out,
                          const double *in, int cb, int dag, void *stream);
int cpsb_mdagm_multi_dev(cpsb_gauge h, const cpsb_dirac_params *p, int precision, int nrhs, double *out,
                         const double *in, double *dot, void *stream);
/* cpsb_minvcg with b and the solutions x[s] in device memory (x: host array of
 * device pointers). */
int cpsb_minvcg_dev(cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a, double *const *x,
                    const double *b, const double *shift, int nshift, double *rsd, int type, const double *alpha,
                    cpsb_solve_result *res, void *stream);
/* Batched DiracOp::MInvCG: nvec source vectors with the same shifts solved
 * together -- the pseudofermions of one RHMC force or action evaluation, which
 * CPS solves one Lattice::FmatEvlMInv call after another
 * (alg/alg_int/alg_action_rational.C:259-359; minvcg.C:47-353 per call).  Every
 * vector keeps its own recurrences, convergence flags and reported residuals,
 * exactly as its own cpsb_minvcg call would; each MatPcDagMatPc is one launch
 * for all vectors that are still iterating, and with a->precision != F64 each
 * shift's refinement is one multi-right-hand-side mixed CG over the vectors.
 * b[q]: the nvec sources.  x[q * nsol + s] (nsol = nshift for CPSB_MULTI, 1 for
 * CPSB_SINGLE): the solutions.  rsd[q * nshift + s]: stop_rsd of shift s for
 * vector q on entry, its reported residual on return.  res[q]: the report of
 * vector q.  nvec <= 16.  Device memory: (nshift + 3) Krylov vectors and nsol
 * solutions per source vector, plus the FP64 inputs and outputs. */
int cpsb_minvcg_multi(cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a, int nvec, double **x,
                      const double *const *b, const double *shift, int nshift, double *rsd, int type,
                      const double *alpha, cpsb_solve_result *res);
/* The same with device vectors: b holds the nvec sources consecutively; x is a
 * host array of device pointers, indexed as above. */
int cpsb_minvcg_multi_dev(cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a, int nvec,
                          double *const *x, const double *b, const double *shift, int nshift, double *rsd, int type,
                          const double *alpha, cpsb_solve_result *res, void *stream);

/* Dslash and MatPcDagMatPc evaluated with fields and links stored in the
 * given precision (CPSB_PREC_F32: FP32 spinors, recon-12 FP32 links;
 * CPSB_PREC_F16: 16-bit fixed-point spinors and links), the operators that
 * the inner solves of mixed-precision InvCg / MInvCG apply.  Same interfaces
 * as cpsb_dslash (DiracWilson::Dslash, d_op_wilson.h:135) and cpsb_mdagm
 * (DiracOp::MatPcDagMatPc, dirac_op.h:198); in and out are FP64 CPS-order host
 * vectors, converted on the device.  CPS has no reduced-precision counterpart. */
int cpsb_dslash_ex(cpsb_gauge h, const cpsb_dirac_params *p, int precision, double *out, const double *in, int cb,
                   int dag);
int cpsb_mdagm_ex(cpsb_gauge h, const cpsb_dirac_params *p, int precision, double *out, const double *in,
                  double *dot);

/* Kernels this library has launched in the process (a graph replay counts each
 * of its kernel nodes): the device analogue of CPS's static flop counter
 * DiracOp::CGflops (include/util/dirac_op.h:74). */
int cpsb_kernel_launches(unsigned long long *count);

/* Times `reps` applications of the device Dslash of the given precision on
 * internally resident data (one checkerboard, dag 0, nrhs right-hand sides of
 * seeded random spinors; consecutive applications cycle through enough field
 * pairs to touch more than twice the L2); reports the mean kernel time in ms
 * measured with CUDA events on the launching stream, and the bytes each
 * application must move (spinors in + out + links).  No counterpart in the
 * reference. */
int cpsb_bench_dslash(cpsb_gauge h, const cpsb_dirac_params *p, int precision, int nrhs, int reps, double *ms,
                      double *bytes);

/* Real parts of nvec dot products <x_v, y_v> of device vectors of n doubles
 * each (vector v starts at x + v*n), written to result[0..nvec) in device
 * memory, in a fixed (reproducible) summation order.  It allocates nothing:
 * for callers that cannot call cudaMalloc -- solvers and HMC loops that run
 * inside an HBM arena they reserved up front and may not grow, and codes that
 * must avoid the device-wide synchronisation of cudaFree.  Its reduction
 * scratch is an 80 KiB file-scope __device__ array that every GPU using the
 * library keeps until exit; the first call on a device looks up that array's
 * device address (make this first call before any stream capture).  Calls
 * whose work overlaps on the GPU share the array and race: serialise them on
 * one stream.  Limits: 1 <= nvec <= 16, n >= 1; larger nvec is rejected with
 * CPSB_ERR_ARG.  Uses the current CUDA device; needs no cpsb_init.  It has no
 * counterpart in the reference. */
int cpsb_redot_noalloc(const double *x, const double *y, long n, int nvec, double *result, void *stream);

/* Request loop for concurrent solves.  CPS runs one DiracOp at a time
 * (DiracOp::scope_lock, d_op_base/comsrc/dirac_op_base.C:26,112-118); a caller
 * that issues many Lattice::FmatEvlInv solves (lattice.h:942) -- differing
 * lattice, Ls, mass, tolerance and right-hand-side count, against gauge fields
 * that stay loaded -- submits them here instead.  No counterpart in the
 * reference.
 *
 * cpsb_serve_create: `slots` worker threads, each with its own CUDA stream,
 *   run admitted solves concurrently.  The HBM budget is hbm_fraction of the
 *   device memory free at creation (0 < hbm_fraction <= 1), capped at
 *   hbm_bytes when nonzero.
 * cpsb_serve_submit: queues the solve of nrhs systems MatPcDagMatPc x = b
 *   (semantics of cpsb_invcg_multi: x holds the guesses on entry).  x[] and
 *   b[] must stay valid until cpsb_serve_wait returns.  The request runs as
 *   work items of up to 16 right-hand sides, each admitted when a slot is free
 *   and its device footprint fits the unreserved budget; a request of which
 *   one right-hand side exceeds the budget returns CPSB_ERR_OOM.
 * cpsb_serve_poll: *done = 1 once every item has finished.
 * cpsb_serve_wait: blocks until the request is done, fills res[nrhs] and the
 *   latency (submission to completion, ms), releases the id and returns the
 *   request's status.
 * cpsb_serve_stats: latency percentiles and throughput of completed requests.
 * cpsb_serve_destroy: serves what is queued, then joins the workers. */
typedef struct cpsb_server_s *cpsb_server;
typedef struct {
  long completed;              /* requests finished with status >= 0 */
  long failed;                 /* requests finished with an error */
  long rhs_completed;          /* right-hand sides of the completed requests */
  double p50_ms, p99_ms, mean_ms, max_ms;
  double requests_per_s;       /* completed / (last completion - first submission) */
  double rhs_per_s;
  int peak_running;            /* most work items running at once */
  int queued, running;
  double budget_bytes, peak_reserved_bytes;
} cpsb_serve_stats_t;
int cpsb_serve_create(cpsb_server *s, int slots, double hbm_fraction, unsigned long long hbm_bytes);
int cpsb_serve_submit(cpsb_server s, cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a, int nrhs,
                      double **x, const double *const *b, unsigned long long *id);
/* Queues a multishift solve (the arguments and results of cpsb_minvcg; x[],
 * b, shift, rsd and alpha must stay valid until cpsb_serve_wait returns, which
 * fills one cpsb_solve_result).  RHMC callers submit the solves of all their
 * pseudofermions (Lattice::FmatEvlMInv per pseudofermion,
 * alg/alg_int/alg_action_rational.C:259-359) and they overlap on the device. */
int cpsb_serve_submit_minvcg(cpsb_server s, cpsb_gauge h, const cpsb_dirac_params *p, const cpsb_cg_arg *a,
                             double **x, const double *b, const double *shift, int nshift, double *rsd, int type,
                             const double *alpha, unsigned long long *id);
int cpsb_serve_poll(cpsb_server s, unsigned long long id, int *done);
int cpsb_serve_wait(cpsb_server s, unsigned long long id, cpsb_solve_result *res, double *latency_ms);
int cpsb_serve_stats(cpsb_server s, cpsb_serve_stats_t *st);
int cpsb_serve_destroy(cpsb_server s);

#ifdef __cplusplus
}
#endif
#endif /* CPSB200_H */
