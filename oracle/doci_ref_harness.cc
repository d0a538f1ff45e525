/*
 * ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * C entry points around hilbert's own v2RDM-DOCI map code (compiled from the
 * reference tree by oracle/build_ref.sh).  The setup below restates only the
 * member initialisation that the reference takes from a Psi4 wavefunction in
 *   src/v2rdm_doci/v2rdm_doci_solver.cc:129-420  (common_init, C1, no frozen
 *                                                 or restricted orbitals)
 *   src/v2rdm_doci/tei.cc:44-125                 (GetIntegrals: packed h and
 *                                                 the 4-index TEI buffer)
 *   src/v2rdm_doci/v2rdm_doci_solver.cc:1058-1074 (compute_energy: Guess,
 *                                                 GetIntegrals, BuildConstraints)
 * Everything else runs the reference's own compiled functions: the sizing,
 * offsets and block list (the POSITIVITY part of common_init, extracted by
 * build_ref.sh), BuildBasis, BuildConstraints, Guess, RepackIntegrals (c),
 * bpsdp_Au, bpsdp_ATu, PackSpatialDensity and WriteTPDM.
 */
#include <cstring>
#include <string>
#include <psi4/psi4-dec.h>
#include <psi4/libqt/qt.h>
#include "v2rdm_doci_solver.h"

using namespace psi;

namespace psi {
std::shared_ptr<PsiOutStream> outfile = std::make_shared<PsiOutStream>();
}

namespace hilbert {

/* members the compiled files reference but the oracle never exercises */
SharedMatrix v2RDM_DOCISolver::GetOEI() { throw PsiException("molecular OEI not available in the oracle", __FILE__, __LINE__); }
void v2RDM_DOCISolver::GetTEIFromDisk() { throw PsiException("disk TEI not available in the oracle", __FILE__, __LINE__); }
double v2RDM_DOCISolver::compute_energy() { throw PsiException("the oracle does not solve", __FILE__, __LINE__); }

v2RDM_DOCISolver::v2RDM_DOCISolver(SharedWavefunction, Options &options) : Wavefunction(options) {}
v2RDM_DOCISolver::~v2RDM_DOCISolver() {}

/* the option set lives as long as the problem (the base class keeps a reference) */
struct OptionHolder {
    Options opts;
};

class RefDoci : private OptionHolder, public v2RDM_DOCISolver {
  public:
    RefDoci(int nmo, int nalpha, int nbeta, const char *positivity, bool d3)
        : OptionHolder(), v2RDM_DOCISolver(nullptr, set(opts, positivity, d3)) {
        nalpha_ = nalpha;
        nbeta_ = nbeta;
        nmo_ = nso_ = nmo;
        nirrep_ = 1;
        is_df_ = false;
        enuc_ = escf_ = efzc_ = 0.0;
        nalphapi_ = Dimension(1);
        nbetapi_ = Dimension(1);
        doccpi_ = Dimension(1);
        soccpi_ = Dimension(1);
        frzcpi_ = Dimension(1);
        frzvpi_ = Dimension(1);
        nmopi_ = Dimension(1);
        nsopi_ = Dimension(1);
        nalphapi_[0] = nalpha;
        nbetapi_[0] = nbeta;
        doccpi_[0] = nbeta;
        soccpi_[0] = nalpha - nbeta;
        nmopi_[0] = nmo;
        nsopi_[0] = nmo;
        rstcpi_ = (int *)calloc(1, sizeof(int));
        rstvpi_ = (int *)calloc(1, sizeof(int));
        amopi_ = (int *)calloc(1, sizeof(int));
        amopi_[0] = nmo;
        amo_ = nmo;
        nfrzc_ = nfrzv_ = nrstc_ = nrstv_ = 0;
        d2_act_spatial_sym_ = d1_act_spatial_sym_ = nullptr;
        epsilon_a_ = std::make_shared<Vector>(nmopi_);
        epsilon_b_ = std::make_shared<Vector>(nmopi_);

        common_init();   // the POSITIVITY / CONSTRAIN_D3 sizing part, extracted

        x = SharedVector(new Vector("primal solution", dimx_));
        c = SharedVector(new Vector("OEI and TEI", dimx_));
        b = SharedVector(new Vector("constraints", nconstraints_));
        Guess();
        BuildConstraints();
    }

    /* GetIntegrals' packing of h (tei.cc:98-106) and of a 4-index (ij|kl)
       buffer in the layout TEI() reads (tei.cc:173-197), then the
       reference's RepackIntegrals */
    void integrals(const double *h, const double *g) {
        const int n = amo_;
        long ntri = (long)n * (n + 1) / 2;
        oei_full_sym_ = (double *)calloc(ntri, sizeof(double));
        for (int i = 0; i < n; i++)
            for (int j = 0; j <= i; j++) oei_full_sym_[INDEX(i, j)] = h[i * n + j];
        tei_full_dim_ = (long)gems_full[0] * (gems_full[0] + 1L) / 2L;
        tei_full_sym_ = (double *)calloc(tei_full_dim_, sizeof(double));
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++)
                for (int k = 0; k < n; k++)
                    for (int l = 0; l < n; l++) {
                        int ij = ibas_full_sym[0][i][j], kl = ibas_full_sym[0][k][l];
                        tei_full_sym_[INDEX(ij, kl)] = g[((long)(i * n + j) * n + k) * n + l];
                    }
        c->zero();
        RepackIntegrals();
    }

    /* PackSpatialDensity (v2rdm_doci_solver.cc:1568-1703) on a given x, with
       the buffers GetIntegrals would allocate (tei.cc:74-94) */
    void alloc_packing() {
        d2_act_spatial_dim_ = gems_00[0] * (gems_00[0] + 1) / 2;
        d1_act_spatial_dim_ = amo_ * (amo_ + 1) / 2;
        free(d2_act_spatial_sym_);
        free(d1_act_spatial_sym_);
        d2_act_spatial_sym_ = (double *)calloc(d2_act_spatial_dim_, sizeof(double));
        d1_act_spatial_sym_ = (double *)calloc(d1_act_spatial_dim_, sizeof(double));
    }
    void pack(const double *xin, double *d2, double *d1) {
        std::memcpy(x->pointer(), xin, sizeof(double) * dimx_);
        alloc_packing();
        PackSpatialDensity();
        std::memcpy(d2, d2_act_spatial_sym_, sizeof(double) * d2_act_spatial_dim_);
        std::memcpy(d1, d1_act_spatial_sym_, sizeof(double) * d1_act_spatial_dim_);
    }
    /* WriteTPDM (src/v2rdm_doci/write_tpdm.cc:47-176) on a given x, into the
       in-memory PSIO stand-in */
    void write_tpdm(const double *xin) {
        std::memcpy(x->pointer(), xin, sizeof(double) * dimx_);
        alloc_packing();
        WriteTPDM();
    }
    long d2_dim() const { return (long)gems_00[0] * (gems_00[0] + 1) / 2; }
    long d1_dim() const { return (long)amo_ * (amo_ + 1) / 2; }

    static Options &set(Options &o, const char *positivity, bool d3) {
        o.set_str("POSITIVITY", positivity);
        o.set_bool("CONSTRAIN_D3", d3);
        return o;
    }

    long n_primal() const { return dimx_; }
    long n_dual() const { return nconstraints_; }
    const std::vector<int> &dims() const { return dimensions_; }
    double *bp() { return b->pointer(); }
    double *cp() { return c->pointer(); }
    double *xp() { return x->pointer(); }
    long block_offset(const std::string &name) const {
        if (name == "d2s2") return d2s2off_;
        if (name == "d2s0") return d2s0off_;
        if (name == "d1") return d1off_;
        if (name == "q2s2") return constrain_q2_ ? q2s2off_ : -1;
        if (name == "q2s0") return constrain_q2_ ? q2s0off_ : -1;
        if (name == "g2s2") return constrain_g2_ ? g2s2off_ : -1;
        if (name == "g2s0") return constrain_g2_ ? g2s0off_ : -1;
        if (name == "d3s3") return constrain_d3_ ? d3s3off_ : -1;
        if (name == "d3s1") return constrain_d3_ ? d3s1off_ : -1;
        if (name == "t1s3aaa") return constrain_t1_ ? t1s3aaaoff_ : -1;
        if (name == "t1s3aab") return constrain_t1_ ? t1s3aaboff_ : -1;
        if (name == "t1s1") return constrain_t1_ ? t1s1off_ : -1;
        if (name == "t2s1") return constrain_t2_ ? t2s1off_ : -1;
        if (name == "t2") return constrain_t2_ ? t2off_ : -1;
        return -2;
    }
};

}  // namespace hilbert

using hilbert::RefDoci;

static thread_local std::string g_err;

extern "C" {

const char *doci_ref_last_error(void) { return g_err.c_str(); }

/* positivity: "D", "DQ", "DG", "DQG", "DQGT1", "DQGT2", "DQGT1T2"; h, g may be NULL */
void *doci_ref_create(int nmo, int nalpha, int nbeta, const char *positivity, int constrain_d3,
                      const double *h, const double *g) {
    try {
        RefDoci *r = new RefDoci(nmo, nalpha, nbeta, positivity, constrain_d3 != 0);
        if (h && g) r->integrals(h, g);
        return r;
    } catch (const std::exception &e) {
        g_err = e.what();
        return nullptr;
    }
}
void doci_ref_destroy(void *p) { delete (RefDoci *)p; }
long doci_ref_n_primal(void *p) { return ((RefDoci *)p)->n_primal(); }
long doci_ref_n_dual(void *p) { return ((RefDoci *)p)->n_dual(); }
int doci_ref_n_blocks(void *p) { return (int)((RefDoci *)p)->dims().size(); }
void doci_ref_block_dims(void *p, int *out) {
    const auto &d = ((RefDoci *)p)->dims();
    std::copy(d.begin(), d.end(), out);
}
long doci_ref_block_offset(void *p, const char *name) { return ((RefDoci *)p)->block_offset(name); }
void doci_ref_get_b(void *p, double *out) {
    RefDoci *r = (RefDoci *)p;
    std::memcpy(out, r->bp(), sizeof(double) * r->n_dual());
}
void doci_ref_get_c(void *p, double *out) {
    RefDoci *r = (RefDoci *)p;
    std::memcpy(out, r->cp(), sizeof(double) * r->n_primal());
}
void doci_ref_get_x(void *p, double *out) {
    RefDoci *r = (RefDoci *)p;
    std::memcpy(out, r->xp(), sizeof(double) * r->n_primal());
}
void doci_ref_Au(void *p, const double *x, double *out) {
    RefDoci *r = (RefDoci *)p;
    std::vector<double> u(x, x + r->n_primal());
    r->bpsdp_Au(out, u.data());
}
long doci_ref_pack_dims(void *p, long *d1n) {
    *d1n = ((RefDoci *)p)->d1_dim();
    return ((RefDoci *)p)->d2_dim();
}
void doci_ref_pack_spatial(void *p, const double *x, double *d2, double *d1) { ((RefDoci *)p)->pack(x, d2, d1); }
void doci_ref_write_tpdm(void *p, const double *x) { ((RefDoci *)p)->write_tpdm(x); }
/* size of one written PSIO entry, -1 if absent; copy it into out (may be NULL) */
long doci_ref_psio_entry(int unit, const char *key, char *out) {
    auto it = psi::psio_store().find({unit, key});
    if (it == psi::psio_store().end()) return -1;
    if (out) std::memcpy(out, it->second.data(), it->second.size());
    return (long)it->second.size();
}
void doci_ref_ATu(void *p, const double *y, double *out) {
    RefDoci *r = (RefDoci *)p;
    std::vector<double> u(y, y + r->n_dual());
    r->bpsdp_ATu(out, u.data());
}

}  // extern "C"
