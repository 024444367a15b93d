/* Test infrastructure only (the checker, never the product).
 *
 * CPU restatement in plain C of the CBS3D++_SI per-step hot path: geometry
 * and boundary preprocessing, greedy element colouring, local time step,
 * LHS diagonals, Steps 1-4, the Jacobi-PCG pressure solve and the
 * convergence norms.  Each function follows the reference file:line cited
 * beside it and keeps its floating-point operation order, so that with
 * -ffp-contract=off on x86-64 every stage is bit-identical to the reference
 * built at -O2 and run with one OpenMP thread.  Arrays are 0-based; node and
 * element ids inside intma/iside stay 1-based as in the reference.
 */
#ifndef CBS_ORACLE_H
#define CBS_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Run configuration: the RunConfig fields the step path reads
 * (include/cbs/core/RunConfig.hpp:38-323). */
typedef struct orc_params {
    int solver_opt, temp_calc, transient_on, dtfixed, ilots, htype, cbs_scheme;
    int step2_check, dtfix_end, convection_type, pnode;
    int dimensional_mode, material_enabled, massflow_enabled;
    int cg_precond, cg_conv_test, cg_max_iter;
    double cinf[5];
    double dtfix, csafm, csafm2, epsilon1, deltr;
    double re, pr, ri;
    double relToler, absToler;
    double heat_flux_bc;
    double outlet_pressure_gauge, inlet_mass_flow_rate, inlet_density, inlet_temperature;
    double inlet_u, inlet_v, inlet_w;
} orc_params;

typedef struct orc_state orc_state;

/* Builds the state from mesh arrays in the reference layout:
 *   intma[4*E]   element-major, 1-based node ids
 *   coord[3*N]   node-major x,y,z
 *   bface[5*NB]  n1 n2 n3 parent solver_bc (raw ids already mapped by .bco)
 *   mat_elem[E]  0 fluid, >0 solid; the five property arrays may be NULL when
 *                material properties are disabled.
 * Runs MeshIO::initialiseFields, the Solver::initialise preprocessing and
 * PressureAssembly::buildElementPressureTerms.  Returns NULL on error and
 * fills err (size errlen). */
orc_state* orc_create(const orc_params* p, int nelem, int npoin, int nboun,
                      const int* intma, const double* coord, const int* bface,
                      const int* mat_elem, const double* rho, const double* cp,
                      const double* k, const double* mu, const double* qvol,
                      char* err, size_t errlen);
void orc_destroy(orc_state* s);

/* One CBS step (src/solver/Solver.cpp:609-680).  0 on success. */
int orc_step(orc_state* s, int iitime);

/* Stage entry points (same order as one step). */
int orc_begin_step(orc_state* s);                 /* unkn1=unkno, pres1=pres, T1=T */
int orc_time_step(orc_state* s, int iitime);      /* TimeStep::computeTimeStep */
int orc_lhs(orc_state* s);                        /* TimeStep::updateLhsDiagonal */
int orc_step1(orc_state* s);                      /* Steps::step1SemiImplicit */
int orc_dt_correction(orc_state* s);              /* TimeStep::applyStep2PressureTimeStepCorrection */
int orc_step2_rhs(orc_state* s);                  /* PressureAssembly::assembleStep2Rhs */
int orc_solve_pressure(orc_state* s);             /* ConjugateGradient::solvePressure + applyPressure */
int orc_step3(orc_state* s);                      /* Steps::step3SemiImplicit */
int orc_step4(orc_state* s);                      /* Steps::step4Energy */
int orc_convergence(orc_state* s);                /* updateVelocityMagnitude + Convergence::evaluate */

/* y = A x with the colour-ordered element-by-element operator
 * (src/linalg/MatrixVectorCalc.cpp:125-205). */
int orc_pressure_multiply(orc_state* s, const double* x, double* y);

/* Named array access: returns the element count of the array (or -1), copies
 * min(count, cap) entries when out != NULL.  dtype is 'd' (double) or 'i'
 * (int) and is written to *dtype when non-NULL. */
long orc_get(orc_state* s, const char* name, void* out, long cap, char* dtype);
/* Overwrites a named double/int array (same names as orc_get). */
int orc_set(orc_state* s, const char* name, const void* in, long count);

const char* orc_error(orc_state* s);

#ifdef __cplusplus
}
#endif
#endif
