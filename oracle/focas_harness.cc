// ORACLE -- test infrastructure only.
//
// Harness for focas's C++ orbital optimizer compiled from the reference
// sources (src/focas/C_files/*.cc, built by oracle/build_ref.sh into
// oracle/_ref/libfocas_ref.so).  The real constructor
// (src/focas/orbital_optimizer.cc:52-376) reads the orbital spaces from a
// Psi4 wavefunction; the constructor here takes them directly for C1
// (ncore restricted doubly occupied, nact active, nvirt restricted virtual
// orbitals, no frozen ones) and makes the same member assignments, then
// sets up the index maps as the real one does (Alloc_OindMap,
// Determine_OindMap).  In C1 the energy order is the orbital order, so every
// orbital_symmetries_ entry is irrep 0.
//
// Also here: the BLAS / LAPACK glue the C_files link against.  hilbert's
// misc/blas.h declares psi::fnocc::F_DGEMM (defined in Psi4's fnocc library:
// a column-major dgemm call) and focas calls libqt's C_DSYEVD; both are
// restated as direct calls of numpy's ILP64 OpenBLAS (64-bit integers).
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <misc/blas.h>

#include "orbital_optimizer.h"

extern "C" {
void scipy_dgemm_64_(const char *ta, const char *tb, const long *m, const long *n, const long *k,
                     const double *alpha, const double *a, const long *lda, const double *b, const long *ldb,
                     const double *beta, double *c, const long *ldc);
void scipy_dsyevd_64_(const char *jobz, const char *uplo, const long *n, double *a, const long *lda, double *w,
                      double *work, const long *lwork, long *iwork, const long *liwork, long *info);
}

namespace psi {
std::shared_ptr<PsiOutStream> outfile = std::make_shared<PsiOutStream>();

namespace fnocc {
void F_DGEMM(char transa, char transb, integer m, integer n, integer k, doublereal alpha, doublereal *A,
             integer lda, doublereal *B, integer ldb, doublereal beta, doublereal *C, integer ldc) {
    scipy_dgemm_64_(&transa, &transb, &m, &n, &k, &alpha, A, &lda, B, &ldb, &beta, C, &ldc);
}
}  // namespace fnocc

int C_DSYEVD(char jobz, char uplo, int n, double *a, int lda, double *w, double *work, int lwork, int *iwork,
             int liwork) {
    const long ln = n, llda = lda, llwork = lwork, lliwork = liwork;
    std::vector<long> iw(std::max(liwork, 1));
    long info = 0;
    scipy_dsyevd_64_(&jobz, &uplo, &ln, a, &llda, w, work, &llwork, iw.data(), &lliwork, &info);
    for (int i = 0; i < liwork; i++) iwork[i] = (int)iw[i];
    return (int)info;
}
}  // namespace psi

namespace hilbert {

struct FocasHarnessSetup {
    int ncore, nact, nvirt;
    long naux;
    bool active_active, exact_diagonal_hessian;
    int maxiter;
    double g_conv, e_conv;
};

OrbitalOptimizer::OrbitalOptimizer(const FocasHarnessSetup &s) {
    is_energy_converged_ = false;
    is_gradient_converged_ = false;
    nirrep_ = 1;
    nmo_ = s.ncore + s.nact + s.nvirt;
    nQ_ = s.naux;
    doccpi_ = Dimension(1);
    frzcpi_ = Dimension(1);
    frzvpi_ = Dimension(1);
    nmopi_ = Dimension(1);
    nmopi_[0] = nmo_;
    rstcpi_ = (int *)malloc(sizeof(int));
    rstvpi_ = (int *)malloc(sizeof(int));
    amopi_ = (int *)malloc(sizeof(int));
    rstcpi_[0] = s.ncore;
    rstvpi_[0] = s.nvirt;
    amopi_[0] = s.nact;
    nfrzc_ = 0;
    nrstc_ = s.ncore;
    nrstv_ = s.nvirt;
    nfrzv_ = 0;
    amo_ = s.nact;
    orbital_symmetries_ = (int *)calloc(nmo_, sizeof(int));
    e_convergence_ = s.e_conv;
    g_convergence_ = s.g_conv;
    active_active_rotations_ = s.active_active;
    maxiter_ = s.maxiter;
    write_ = false;
    exact_diagonal_hessian_ = s.exact_diagonal_hessian;
    algorithm_ = "";
    oo_active_active_rotations_ = active_active_rotations_;
    oo_maxiter_ = maxiter_;
    oo_energy_convergence_ = e_convergence_;
    oo_gradient_convergence_ = g_convergence_;
    oo_exact_diagonal_hessian_ = exact_diagonal_hessian_;
    Alloc_OindMap();
    Determine_OindMap();
}

OrbitalOptimizer::~OrbitalOptimizer() {
    free(rstcpi_);
    free(rstvpi_);
    free(amopi_);
    free(orbital_symmetries_);
    Dealloc_OindMap();
}

struct FocasHarness {
    // gradient, diagonal Hessian and energy at the current orbitals; d2, d1
    // and oei are sorted in and back out around the evaluation, as
    // optimize_orbitals does
    static double egh(OrbitalOptimizer &o, double *d2, double *d1, double *tei, double *oei, double *U,
                      double *grad, double *hdiag, double *gnorm) {
        o.Initiate_Optimizer(d2, d1, oei, U);
        const double E = o.Compute_EGH(d2, d1, tei, oei);
        std::memcpy(grad, o.orbital_gradient_, o.Nrot_ * sizeof(double));
        std::memcpy(hdiag, o.diagonal_orbital_hessian_, o.Nrot_ * sizeof(double));
        *gnorm = o.gradient_norm_;
        o.Finalize_Optimizer(d2, d1, oei, U);
        return E;
    }
    static int nrot(OrbitalOptimizer &o, double *d2, double *d1, double *oei, double *U) {
        o.Initiate_Optimizer(d2, d1, oei, U);
        const int n = o.Nrot_;
        o.Finalize_Optimizer(d2, d1, oei, U);
        return n;
    }
};

}  // namespace hilbert

using hilbert::FocasHarness;
using hilbert::FocasHarnessSetup;
using hilbert::OrbitalOptimizer;

extern "C" {

void *v2b_focas_create(int ncore, int nact, int nvirt, long naux, int active_active, int exact_diagonal_hessian,
                       int maxiter, double g_conv, double e_conv) {
    FocasHarnessSetup s{ncore, nact, nvirt, naux, active_active != 0, exact_diagonal_hessian != 0, maxiter,
                        g_conv, e_conv};
    return new OrbitalOptimizer(s);
}

void v2b_focas_destroy(void *h) { delete (OrbitalOptimizer *)h; }

int v2b_focas_nrot(void *h, double *d2, double *d1, double *oei, double *U) {
    return FocasHarness::nrot(*(OrbitalOptimizer *)h, d2, d1, oei, U);
}

double v2b_focas_egh(void *h, double *d2, double *d1, double *tei, double *oei, double *U, double *grad,
                     double *hdiag, double *gnorm) {
    return FocasHarness::egh(*(OrbitalOptimizer *)h, d2, d1, tei, oei, U, grad, hdiag, gnorm);
}

// OrbitalOptimizer::optimize_orbitals (orbopt_optimize.cc:25-98): tei, oei
// and the transformation matrix U are updated in place
void v2b_focas_optimize(void *h, double *d2, double *d1, double *tei, double *oei, double *U, double *dE,
                        double *gnorm, int *iter) {
    ((OrbitalOptimizer *)h)->optimize_orbitals(d2, d1, tei, oei, U, *dE, *gnorm, *iter);
}
}
