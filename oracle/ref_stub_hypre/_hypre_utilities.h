/* Stand-in for the HYPRE headers, used only to compile the reference's
 * HypreFDM 3D solver (HelmholtzSolvers/HypreFDM/src/Helmholtz3D_MPI.cpp) into
 * the oracle's reference library under oracle/_ref.
 *
 * Test infrastructure: the product never includes this header.
 *
 * It keeps the IJ interface the solver assembles through
 * (Helmholtz3D_MPI.cpp:258-275 create/destroy, :299-418 the matrix rows,
 * :428-490 the right-hand side and the initial guess) as plain in-memory
 * objects: a matrix is one sparse row per global index with HYPRE's "set"
 * semantics (a value replaces an earlier one of the same column), a vector is
 * a dense array over its index range.  ParCSR objects are the same objects.
 * The Krylov solve itself (HypreSolvers.cpp) is not compiled; the driver
 * oracle/ref_driver_fd3d.cpp supplies HypreSolve as a direct solve of the
 * assembled system.
 */
#ifndef ORACLE_STUB_HYPRE_H
#define ORACLE_STUB_HYPRE_H
#include <map>
#include <vector>

#include "mpi.h"

struct oracle_ij_matrix {
    int lo = 0, hi = -1;
    std::vector<std::map<int, double>> rows;
};
struct oracle_ij_vector {
    int lo = 0, hi = -1;
    std::vector<double> v;
};
typedef oracle_ij_matrix* HYPRE_IJMatrix;
typedef oracle_ij_matrix* HYPRE_ParCSRMatrix;
typedef oracle_ij_vector* HYPRE_IJVector;
typedef oracle_ij_vector* HYPRE_ParVector;
typedef int HYPRE_Int;
typedef int HYPRE_BigInt;
typedef double HYPRE_Complex;
typedef void* HYPRE_Solver;
#define HYPRE_PARCSR 5555

static inline int HYPRE_IJMatrixCreate(MPI_Comm, int ilo, int ihi, int, int, HYPRE_IJMatrix* m)
{
    *m = new oracle_ij_matrix;
    (*m)->lo = ilo;
    (*m)->hi = ihi;
    (*m)->rows.assign(ihi >= ilo ? ihi - ilo + 1 : 0, {});
    return 0;
}
static inline int HYPRE_IJMatrixSetObjectType(HYPRE_IJMatrix, int) { return 0; }
static inline int HYPRE_IJMatrixInitialize(HYPRE_IJMatrix) { return 0; }
static inline int HYPRE_IJMatrixSetValues(HYPRE_IJMatrix m, int nrows, int* ncols, const int* rows, const int* cols,
                                          const double* values)
{
    int at = 0;
    for (int r = 0; r < nrows; ++r)
        for (int c = 0; c < ncols[r]; ++c, ++at) m->rows[rows[r] - m->lo][cols[at]] = values[at];
    return 0;
}
static inline int HYPRE_IJMatrixAssemble(HYPRE_IJMatrix) { return 0; }
static inline int HYPRE_IJMatrixGetObject(HYPRE_IJMatrix m, void** obj)
{
    *obj = m;
    return 0;
}
static inline int HYPRE_IJMatrixDestroy(HYPRE_IJMatrix m)
{
    delete m;
    return 0;
}

static inline int HYPRE_IJVectorCreate(MPI_Comm, int lo, int hi, HYPRE_IJVector* v)
{
    *v = new oracle_ij_vector;
    (*v)->lo = lo;
    (*v)->hi = hi;
    (*v)->v.assign(hi >= lo ? hi - lo + 1 : 0, 0.0);
    return 0;
}
static inline int HYPRE_IJVectorSetObjectType(HYPRE_IJVector, int) { return 0; }
static inline int HYPRE_IJVectorInitialize(HYPRE_IJVector) { return 0; }
static inline int HYPRE_IJVectorSetValues(HYPRE_IJVector v, int n, const int* idx, const double* values)
{
    for (int i = 0; i < n; ++i) v->v[idx[i] - v->lo] = values[i];
    return 0;
}
static inline int HYPRE_IJVectorGetValues(HYPRE_IJVector v, int n, const int* idx, double* values)
{
    for (int i = 0; i < n; ++i) values[i] = v->v[idx[i] - v->lo];
    return 0;
}
static inline int HYPRE_IJVectorAssemble(HYPRE_IJVector) { return 0; }
static inline int HYPRE_IJVectorGetObject(HYPRE_IJVector v, void** obj)
{
    *obj = v;
    return 0;
}
static inline int HYPRE_IJVectorDestroy(HYPRE_IJVector v)
{
    delete v;
    return 0;
}
#endif
