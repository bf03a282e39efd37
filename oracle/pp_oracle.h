/*
 * pp_oracle.h -- CPU restatement of PittPack's single-rank Poisson solve.
 * TEST INFRASTRUCTURE ONLY (the checker); the product never includes it.
 */
#ifndef PP_ORACLE_H
#define PP_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
    PPO_BAD = -1,
    PPO_DST2 = 0, /* D-D: DST-II forward / DST-III inverse (reference tag 0) */
    PPO_DCT2 = 1, /* N-N: DCT-II / DCT-III (reference tag 1) */
    PPO_FFT = 2,  /* P-P: complex DFT (reference tag 2) */
    PPO_DCT4 = 3, /* N-D: DCT-IV (not in the reference) */
    PPO_DST4 = 4  /* D-N: DST-IV (not in the reference) */
};

#define PPO_ERR_INPUT 19 /* the reference's INPUT_ARGS code */

typedef struct {
    int nx, ny, nz;
    char bc[6];          /* xmin xmax ymin ymax zmin zmax, letters P N D */
    double box[6];       /* Xa Xb Ya Yb Za Zb */
    int compat_zero_mode; /* 1: the reference's zero-mode row replacement */
    int dirichlet_lift;   /* 1: the reference's modifyRhsDirichlet */
    /* caller's boundary data per face (order of bc; NULL: none): Dirichlet
     * values or Neumann outward derivatives at the face's cell centres, x
     * faces [j + ny k], y faces [i + nx k], z faces [i + nx j]; a face with
     * data takes no manufactured lift.  Not in the reference: the ghost-cell
     * relations u_g = 2 g - u_0 (D) and u_g = u_0 + h g (N) with the face's
     * stencil weight (dz/dx)^2, (dz/dy)^2 or 1. */
    const double* face[6];
    int zero_mean;        /* 1: the reference's ZERO_MEAN (subtractMeanValue) */
    /* the reference's SOLUTIONMETHOD (src/pencilDcmp.cpp:6102-6148): 0 Thomas
     * (default), 1 its normalised PCR, 2 its CR-P, as its CPU build computes
     * them (ppo_check gives the sizes each is defined for) */
    int z_method;
} ppo_problem;

int ppo_kind_from_bc(char lo, char hi);
int ppo_check(const ppo_problem* pb);
int ppo_ref_pcr_defined(int nz, char z0, char z1);
int ppo_ref_crp_defined(int nz, char z0, char z1);
double ppo_eigenvalue(const ppo_problem* pb, int kx, int ky);
void ppo_dft(int n, int sign, double* re, double* im);
void ppo_dirichlet_lift(const ppo_problem* pb, double* lift);
/* P: 2*nx*ny*nz doubles, chunkedArray layout P[2*(i+nx*j+nx*ny*k)+{0,1}] */
int ppo_solve(const ppo_problem* pb, const double* rhs_re, const double* rhs_im, double* P);
void ppo_manufactured(const ppo_problem* pb, double* f_re, double* f_im, double* u_re, double* u_im);
void ppo_residual(const ppo_problem* pb, const double* u, const double* b, double* r);

#ifdef __cplusplus
}
#endif
#endif
