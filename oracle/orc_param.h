/*
 * orc_param.h -- flat run-parameter record shared by the two CPU checkers
 * (oracle/hydro_oracle.c, the restatement, and oracle/ref_shim.c, the harness
 * around the reference's own objects).  TEST INFRASTRUCTURE ONLY.
 * Field meaning follows hydroparam_t (HydroC99_2Domp/Src/parametres.h:31-80).
 */
#ifndef ORC_PARAM_H
#define ORC_PARAM_H
typedef struct {
    int nx, ny;
    int boundary_left, boundary_right, boundary_down, boundary_up;
    int iorder;
    int scheme; /* 1 muscl, 2 plmde, 3 collela */
    int niter_riemann;
    double slope_type, gamma, smallr, smallc, dx, courant_factor;
} orc_param_t;
#endif
