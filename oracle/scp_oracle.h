/* scp_oracle.h -- CPU restatement of the reference's complex / gauged lattice
 * stepper (kardianos/scp sfa/sim/scp_sim.c), used ONLY as the checker of the
 * parity tests, smoke() and the CPU-baseline leg of bench.py.  Nothing in the
 * product links, loads or calls it.
 *
 * Column order of every state array passed in or out (the SFA snapshot
 * registration order of sfa/sim/scp_sim.c:2862-2897):
 *    0- 2 phi_{x,y,z}      (u_a = Re Phi_a)
 *    3- 5 theta_{x,y,z}    (tu_a = Re Theta_a)
 *    6- 8 phi_v{x,y,z}     (du_a/dt)
 *    9-11 theta_v{x,y,z}   (dtu_a/dt)
 *   12-14 phiim_{x,y,z}    (v_a = Im Phi_a)
 *   15-17 thetaim_{x,y,z}  (tv_a = Im Theta_a)
 *   18-20 phiim_v{x,y,z}
 *   21-23 thetaim_v{x,y,z}
 *   24-26 th_{x,y,z}       (link angles, gauged only)
 *   27-29 E_{x,y,z}        (link electric field, gauged only)
 *   30-35 th2_*, E2_*      (orc_get only, second gauge on)
 * Three fabrics: orc_create takes 30 + 24 (Q) + 24 (L) columns, orc_get
 * returns the 30 of C and the 24 of L (the reference's archive schema).
 *
 * Diagnostic slots (orc_diag) follow the reference diag TSV column order
 * (sfa/sim/scp_sim.c:2993-3003) without the leading time column; see
 * SCP_DIAG_* in include/scp_gpu.h, which uses the same numbering.
 */
#ifndef SCP_ORACLE_H
#define SCP_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int N;
    double L, dx, dt;
    double m2, mtheta2, eta, mu, kappa;
    int gauge;          /* complex_gauge with g != 0 */
    double g;           /* g_gauge */
    int bc_type;        /* 0 absorbing sphere, 2 periodic */
    double damp_width, damp_rate;
    double qdiag_radius, qdiag_probe1, qdiag_probe2;
    /* gauged extensions (gauge = 1 only; all zero = off): Higgs condensate
     * (higgs_v > 0) and second compact U(1) gauge (g2 != 0, charges q2[]);
     * three matter fabrics (n_fabrics = 3, EM charges q_fab[] = q_C, q_Q, q_L,
     * mf_lock = 1 keeps Q a copy of C as the reference does) */
    double higgs_v, higgs_lam, higgs_kap, higgs_rvoid;
    double g2;
    double q2[3];
    int n_fabrics, mf_lock;
    double q_fab[3];
    /* real 6-field mode (complex_phi = 0, gauge = 0): 12 columns (0-11 of the
     * order above); its optional terms as the reference's Config names them */
    int real_fields, mode;
    double inv_alpha, inv_beta, kappa_gamma, alpha_cs, beta_h, kappa_h;
} orc_params;

typedef struct orc_state orc_state;

/* Allocates the state, copies the 24/30 columns in, and (gauged) runs the
 * net-charge check when bc_type==2 and the one-time Gauss projection, then the
 * initial force evaluation -- the start-up sequence of scp_sim.c main
 * (:2806-2836).  Returns NULL on failure; *status gets a negative code
 * (-1 bad params, -2 net charge, -3 CG did not converge, -4 alloc). */
orc_state *orc_create(const orc_params *p, const double *const *cols, int project, int *status);
void orc_free(orc_state *s);
void orc_step(orc_state *s, int nsteps);
void orc_get(const orc_state *s, double *const *cols);
/* 31 diagnostics in TSV order (see header comment), then Q_C, Q_Q, Q_L,
 * Q_em with three fabrics (35); the real mode's 13 (energies, amplitudes,
 * theta_rms); returns the slot count */
int orc_diag(orc_state *s, double *out);
double orc_g_offset(const orc_state *s);
int orc_cg_iterations(const orc_state *s);
/* accelerations of the current positions: 24 arrays in column order
 * 0-2 phi_acc, 3-5 theta_acc, 6-8 phiim_acc, 9-11 thetaim_acc, and E_acc 12-14 */
void orc_accelerations(orc_state *s, double *const *acc);
/* random lattice gauge transform KAT of scp_sim.c:2461-2556; returns the
 * worst relative deviation over the 10 invariants (<=1e-12 passes) */
double orc_gauge_xform_test(orc_state *s, double *rel_out10);
int orc_threads(void);

#ifdef __cplusplus
}
#endif
#endif
