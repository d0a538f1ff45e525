/*
 * ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * C entry points around hilbert's own v2RDMSolver map code (compiled from the
 * reference tree by oracle/build_ref.sh).  The setup below restates only the
 * member initialisation that the reference performs in
 *   src/v2rdm_casscf/v2rdm_solver.cc:839-962  (initialize_with_hubbard_hamiltonian)
 *   src/v2rdm_casscf/v2rdm_solver.cc:964-1085 (initialize_with_external_hamiltonian)
 *   src/v2rdm_casscf/v2rdm_solver.cc:147-195  (external-Hamiltonian constructor: h, g -> c)
 *   src/v2rdm_casscf/v2rdm_solver.cc:1087-1107 (initialize_common_elements call order)
 *   src/v2rdm_casscf/v2rdm_solver.cc:1272-1292 (compute_energy: Guess, GetIntegrals, BuildConstraints)
 * Everything else (index tables, block sizes, offsets, b, c repacking, guess,
 * A.x and A^T.y) runs the reference's own compiled functions.
 */
#include <cstring>
#include <psi4/psi4-dec.h>
#include <psi4/libqt/qt.h>
#include "v2rdm_solver.h"

using namespace psi;

namespace psi {
std::shared_ptr<PsiOutStream> outfile = std::make_shared<PsiOutStream>();
}

namespace hilbert {

/* members the compiled files reference but the oracle never exercises */
SharedMatrix v2RDMSolver::GetOEI() { throw PsiException("molecular OEI not available in the oracle", __FILE__, __LINE__); }
void v2RDMSolver::GetTEIFromDisk() { throw PsiException("disk TEI not available in the oracle", __FILE__, __LINE__); }
void v2RDMSolver::add_gpc_constraints(int, int) { throw PsiException("GPC not available in the oracle", __FILE__, __LINE__); }
void v2RDMSolver::Generalized_Pauli_constraints_Au(double *, double *, int) { throw PsiException("GPC not available", __FILE__, __LINE__); }
void v2RDMSolver::Generalized_Pauli_constraints_ATu(double *, double *, int) { throw PsiException("GPC not available", __FILE__, __LINE__); }
double v2RDMSolver::compute_energy() { throw PsiException("the oracle does not solve", __FILE__, __LINE__); }

v2RDMSolver::v2RDMSolver(int nalpha, int nbeta, int nmo, std::vector<double>, std::vector<double>,
                         Options &options)
    : Wavefunction(options) {
    nalpha_ = nalpha;
    nbeta_ = nbeta;
    nmo_ = nmo;
    nso_ = nmo;
}
v2RDMSolver::~v2RDMSolver() {}

/* thin subclass: gives the C entry points access to the protected state */
class RefProblem : public v2RDMSolver {
  public:
    RefProblem(int nmo, int nalpha, int nbeta, bool hubbard, const double *h, const double *g,
               Options &opts)
        : v2RDMSolver(nalpha, nbeta, nmo, {}, {}, opts) {
        is_hubbard_ = hubbard;
        is_external_hamiltonian_ = !hubbard;
        is_df_ = false;
        enuc_ = 0.0;
        escf_ = 0.0;
        efzc_ = 0.0;
        amo_ = nmo_;
        nfrzc_ = nfrzv_ = nrstc_ = nrstv_ = 0;
        int ms = (int)nalpha_ - (int)nbeta_;
        multiplicity_ = hubbard ? 2 * ms + 1 : ms + 1;
        nirrep_ = 1;
        nalphapi_ = Dimension(1);
        nbetapi_ = Dimension(1);
        doccpi_ = Dimension(1);
        soccpi_ = Dimension(1);
        frzcpi_ = Dimension(1);
        frzvpi_ = Dimension(1);
        nmopi_ = Dimension(1);
        nsopi_ = Dimension(1);
        rstcpi_ = (int *)calloc(1, sizeof(int));
        rstvpi_ = (int *)calloc(1, sizeof(int));
        amopi_ = (int *)calloc(1, sizeof(int));
        nalphapi_[0] = (int)nalpha_;
        nbetapi_[0] = (int)nbeta_;
        doccpi_[0] = (int)nalpha_;
        soccpi_[0] = 0;
        nmopi_[0] = nmo_;
        nsopi_[0] = nso_;
        amopi_[0] = nmo_;
        epsilon_a_ = std::make_shared<Vector>(nmopi_);
        epsilon_b_ = std::make_shared<Vector>(nmopi_);

        set_constraints();
        build_mapping_arrays();
        determine_n_primal();
        determine_n_dual();
        set_primal_offsets();

        x = SharedVector(new Vector("primal solution", n_primal_));
        c = SharedVector(new Vector("OEI and TEI", n_primal_));
        b = SharedVector(new Vector("constraints", n_dual_));

        if (!hubbard) {
            double *c_p = c->pointer();
            for (int i = 0; i < amo_; i++)
                for (int j = 0; j < amo_; j++) {
                    c_p[d1aoff[0] + i * amo_ + j] = h[i * amo_ + j];
                    c_p[d1boff[0] + i * amo_ + j] = h[i * amo_ + j];
                }
            long n = amo_;
            for (int ij = 0; ij < gems_ab[0]; ij++) {
                long i = bas_ab_sym[0][ij][0], j = bas_ab_sym[0][ij][1];
                for (int kl = 0; kl < gems_ab[0]; kl++) {
                    long k = bas_ab_sym[0][kl][0], l = bas_ab_sym[0][kl][1];
                    c_p[d2aboff[0] + ij * gems_ab[0] + kl] = g[i * n * n * n + k * n * n + j * n + l];
                }
            }
            for (int ij = 0; ij < gems_aa[0]; ij++) {
                long i = bas_aa_sym[0][ij][0], j = bas_aa_sym[0][ij][1];
                for (int kl = 0; kl < gems_aa[0]; kl++) {
                    long k = bas_aa_sym[0][kl][0], l = bas_aa_sym[0][kl][1];
                    double val = g[i * n * n * n + k * n * n + j * n + l] - g[i * n * n * n + l * n * n + j * n + k];
                    c_p[d2aaoff[0] + ij * gems_aa[0] + kl] = val;
                    c_p[d2bboff[0] + ij * gems_aa[0] + kl] = val;
                }
            }
        }
        Guess();
        GetIntegrals();
        BuildConstraints();
    }

    long np() const { return n_primal_; }
    long nd() const { return n_dual_; }
    const std::vector<int> &dims() const { return dimensions_; }
    double *bp() { return b->pointer(); }
    double *cp() { return c->pointer(); }
    double *xp() { return x->pointer(); }
    // v2rdm_solver.cc:3110-3219 on a given primal vector
    void pack(const double *xin, double *d2, double *d1) {
        std::memcpy(x->pointer(), xin, sizeof(double) * n_primal_);
        PackSpatialDensity();
        std::memcpy(d2, d2_act_spatial_sym_, sizeof(double) * d2_act_spatial_dim_);
        std::memcpy(d1, d1_act_spatial_sym_, sizeof(double) * d1_act_spatial_dim_);
    }
    // write_tpdm.cc:40-519 and write_opdm.cc:40-114 on a given primal vector,
    // into the in-memory PSIO stand-in
    // the writers on a given x; with ncore > 0 they see the C1 orbital
    // numbering build_mapping_arrays gives restricted doubly occupied
    // orbitals (basis.cc:100-111, 415-424): core 0 .. ncore-1, active i at ncore + i
    void write_rdms(const double *xin, int ncore) {
        std::memcpy(x->pointer(), xin, sizeof(double) * n_primal_);
        const int saved_rst = rstcpi_[0], saved_nrst = nrstc_, saved_off = pitzer_offset_full[0];
        std::vector<int> saved_full(full_basis, full_basis + amo_);
        rstcpi_[0] = ncore;
        nrstc_ = ncore;
        pitzer_offset_full[0] = 0;
        for (int i = 0; i < amo_; i++) full_basis[i] = ncore + i;
        WriteTPDM();
        WriteTPDMSpinFree();
        WriteOPDM();
        WriteTPDM_IWL();   // write_tpdm_iwl.cc:45-205, into the IWL stand-in
        if (constrain_d3_) WriteActive3PDM();   // write_3pdm.cc:50-206
        rstcpi_[0] = saved_rst;
        nrstc_ = saved_nrst;
        pitzer_offset_full[0] = saved_off;
        std::copy(saved_full.begin(), saved_full.end(), full_basis);
    }
    long d2_dim() const { return d2_act_spatial_dim_; }
    long d1_dim() const { return d1_act_spatial_dim_; }
    double efzc() const { return efzc_; }

    long block_offset(const std::string &name) const {
        const std::map<std::string, int *> m = {
            {"d2ab", d2aboff}, {"d2aa", d2aaoff}, {"d2bb", d2bboff}, {"d200", d200off},
            {"d1a", d1aoff},   {"d1b", d1boff},   {"q1a", q1aoff},   {"q1b", q1boff},
            {"q2ab", q2aboff}, {"q2aa", q2aaoff}, {"q2bb", q2bboff}, {"g2ab", g2aboff},
            {"g2ba", g2baoff}, {"g2aa", g2aaoff}, {"t2aaa", t2aaaoff}, {"t2bbb", t2bbboff},
            {"t2aab", t2aaboff}, {"t2bba", t2bbaoff}, {"t1aaa", t1aaaoff}, {"t1bbb", t1bbboff},
            {"t1aab", t1aaboff}, {"t1bba", t1bbaoff}, {"d3aaa", d3aaaoff}, {"d3bbb", d3bbboff},
            {"d3aab", d3aaboff}, {"d3bba", d3bbaoff}, {"q3aaa", q3aaaoff}, {"q3bbb", q3bbboff},
            {"q3aab", q3aaboff}, {"q3bba", q3bbaoff}, {"e3aaa", e3aaaoff}, {"e3bbb", e3bbboff},
            {"e3aab", e3aaboff}, {"e3bba", e3bbaoff}, {"f3aaa", f3aaaoff}, {"f3bbb", f3bbboff},
            {"f3aab", f3aaboff}, {"f3bba", f3bbaoff}, {"d4aaaa", d4aaaaoff}, {"d4aaab", d4aaaboff},
            {"d4aabb", d4aabboff}, {"d4bbba", d4bbbaoff}, {"d4bbbb", d4bbbboff}};
        auto it = m.find(name);
        if (it == m.end()) return -1;
        bool present = false;
        if (name == "d200") present = constrain_spin_;
        else if (name[0] == 'q' && name[1] == '2') present = constrain_q2_;
        else if (name[0] == 'g') present = constrain_g2_;
        else if (name[0] == 't' && name[1] == '2') present = constrain_t2_;
        else if (name[0] == 't' && name[1] == '1') present = constrain_t1_;
        else if (name[0] == 'd' && name[1] == '3') present = constrain_d3_;
        else if (name[0] == 'q' && name[1] == '3') present = constrain_q3_;
        else if (name[0] == 'e' && name[1] == '3') present = constrain_e3_;
        else if (name[0] == 'f' && name[1] == '3') present = constrain_f3_;
        else if (name[0] == 'd' && name[1] == '4') present = constrain_d4_;
        else present = true;
        if (!present || it->second == nullptr) return -1;
        return it->second[0];
    }
    int gab() const { return gems_ab[0]; }
    int gaa() const { return gems_aa[0]; }
    void tables(int *bas_ab, int *ibas_ab, int *bas_aa, int *ibas_aa) const {
        for (int n = 0; n < gems_ab[0]; n++) { bas_ab[2 * n] = bas_ab_sym[0][n][0]; bas_ab[2 * n + 1] = bas_ab_sym[0][n][1]; }
        for (int n = 0; n < gems_aa[0]; n++) { bas_aa[2 * n] = bas_aa_sym[0][n][0]; bas_aa[2 * n + 1] = bas_aa_sym[0][n][1]; }
        for (int i = 0; i < amo_; i++)
            for (int j = 0; j < amo_; j++) {
                ibas_ab[i * amo_ + j] = ibas_ab_sym[0][i][j];
                ibas_aa[i * amo_ + j] = ibas_aa_sym[0][i][j];
            }
    }
    void triplet_sizes(int *aaa, int *aab, int *aba) const {
        *aaa = constrain_t2_ || constrain_t1_ || constrain_d3_ ? trip_aaa[0] : 0;
        *aab = constrain_t2_ || constrain_t1_ || constrain_d3_ ? trip_aab[0] : 0;
        *aba = constrain_t2_ || constrain_t1_ || constrain_d3_ ? trip_aba[0] : 0;
    }
};

}  // namespace hilbert

using hilbert::RefProblem;

static thread_local std::string g_last_error;

extern "C" {

const char *v2b_ref_last_error() { return g_last_error.c_str(); }

/* positivity: "D", "DQ", "DG", "DQG", "DQGT1", "DQGT2", "DQGT1T2", optionally followed by
 * "+D3", "+Q3", "+E3", "+F3", "+D4" (CONSTRAIN_D3 / _Q3 / _E3 / _F3 / _D4); guess_hf: 0 random, 1 HF */
void *v2b_ref_create(int nmo, int nalpha, int nbeta, const char *positivity, int constrain_spin,
                     int constrain_sz, int hubbard, double hub_t, double hub_u, const double *h,
                     const double *g, int guess_hf) {
    try {
        auto *opts = new Options();
        std::string pos(positivity);
        bool d3 = false, q3 = false, e3 = false, f3 = false, d4 = false;
        size_t plus = pos.find('+');
        const std::string base = pos.substr(0, plus);
        while (plus != std::string::npos) {
            const size_t next = pos.find('+', plus + 1);
            const std::string tok = pos.substr(plus + 1, next == std::string::npos ? std::string::npos : next - plus - 1);
            if (tok == "D3") d3 = true;
            else if (tok == "Q3") q3 = true;
            else if (tok == "E3") e3 = true;
            else if (tok == "F3") f3 = true;
            else if (tok == "D4") d4 = true;
            else throw std::invalid_argument("unknown constraint suffix");
            plus = next;
        }
        opts->set_str("POSITIVITY", base);
        opts->set_bool("CONSTRAIN_D3", d3);
        opts->set_bool("CONSTRAIN_Q3", q3);
        opts->set_bool("CONSTRAIN_E3", e3);
        opts->set_bool("CONSTRAIN_F3", f3);
        opts->set_bool("CONSTRAIN_D4", d4);
        opts->set_bool("CONSTRAIN_SPIN", constrain_spin != 0);
        opts->set_bool("CONSTRAIN_SZ", constrain_sz != 0);
        opts->set_str("GPC_CONSTRAINTS", "NONE");
        opts->set_bool("HUBBARD_HAMILTONIAN", hubbard != 0);
        opts->set_double("HUBBARD_T", hub_t);
        opts->set_double("HUBBARD_U", hub_u);
        opts->set_str("TPDM_GUESS", guess_hf ? "HF" : "RANDOM");
        return new RefProblem(nmo, nalpha, nbeta, hubbard != 0, h, g, *opts);
    } catch (const std::exception &e) {
        g_last_error = e.what();
        return nullptr;
    }
}
void v2b_ref_destroy(void *p) { delete static_cast<RefProblem *>(p); }
long v2b_ref_n_primal(void *p) { return static_cast<RefProblem *>(p)->np(); }
long v2b_ref_n_dual(void *p) { return static_cast<RefProblem *>(p)->nd(); }
int v2b_ref_n_blocks(void *p) { return (int)static_cast<RefProblem *>(p)->dims().size(); }
void v2b_ref_block_dims(void *p, int *out) {
    const auto &d = static_cast<RefProblem *>(p)->dims();
    for (size_t i = 0; i < d.size(); i++) out[i] = d[i];
}
long v2b_ref_block_offset(void *p, const char *name) { return static_cast<RefProblem *>(p)->block_offset(name); }
void v2b_ref_get_b(void *p, double *out) {
    auto *r = static_cast<RefProblem *>(p);
    std::memcpy(out, r->bp(), sizeof(double) * r->nd());
}
void v2b_ref_get_c(void *p, double *out) {
    auto *r = static_cast<RefProblem *>(p);
    std::memcpy(out, r->cp(), sizeof(double) * r->np());
}
void v2b_ref_get_x(void *p, double *out) {
    auto *r = static_cast<RefProblem *>(p);
    std::memcpy(out, r->xp(), sizeof(double) * r->np());
}
double v2b_ref_efzc(void *p) { return static_cast<RefProblem *>(p)->efzc(); }
int v2b_ref_Au(void *p, double *out, const double *in) {
    try {
        static_cast<RefProblem *>(p)->bpsdp_Au(out, const_cast<double *>(in));
        return 0;
    } catch (const std::exception &e) { g_last_error = e.what(); return 1; }
}
int v2b_ref_ATu(void *p, double *out, const double *in) {
    try {
        static_cast<RefProblem *>(p)->bpsdp_ATu(out, const_cast<double *>(in));
        return 0;
    } catch (const std::exception &e) { g_last_error = e.what(); return 1; }
}
void v2b_ref_gems(void *p, int *gab, int *gaa) {
    *gab = static_cast<RefProblem *>(p)->gab();
    *gaa = static_cast<RefProblem *>(p)->gaa();
}
void v2b_ref_tables(void *p, int *bas_ab, int *ibas_ab, int *bas_aa, int *ibas_aa) {
    static_cast<RefProblem *>(p)->tables(bas_ab, ibas_ab, bas_aa, ibas_aa);
}
void v2b_ref_triplets(void *p, int *aaa, int *aab, int *aba) {
    static_cast<RefProblem *>(p)->triplet_sizes(aaa, aab, aba);
}

long v2b_ref_pack_dims(void *p, long *d1n) {
    *d1n = static_cast<RefProblem *>(p)->d1_dim();
    return static_cast<RefProblem *>(p)->d2_dim();
}
/* runs the reference's RDM writers on x; their files stay in the PSIO
   stand-in until the next call */
int v2b_ref_write_rdms(void *p, const double *x, int ncore) {
    try {
        static_cast<RefProblem *>(p)->write_rdms(x, ncore);
        return 0;
    } catch (const std::exception &e) { g_last_error = e.what(); return 1; }
}
/* the write_value calls of the IWL writer on one file ("aa", "ab", "bb"):
   their count, copied into out (5 doubles each: p, q, r, s, value) if not
   NULL; *cutoff receives the file's cutoff */
long v2b_ref_iwl_records(const char *spin, double *out, double *cutoff) {
    const int unit = spin[1] == 'b' ? (spin[0] == 'a' ? PSIF_MO_AB_TPDM : PSIF_MO_BB_TPDM) : PSIF_MO_AA_TPDM;
    auto it = psi::iwl_store().find(unit);
    if (it == psi::iwl_store().end()) return -1;
    if (cutoff) *cutoff = it->second.cutoff;
    const auto &rec = it->second.records;
    if (out)
        for (size_t k = 0; k < rec.size(); k++) {
            out[5 * k] = rec[k].p; out[5 * k + 1] = rec[k].q; out[5 * k + 2] = rec[k].r;
            out[5 * k + 3] = rec[k].s; out[5 * k + 4] = rec[k].value;
        }
    return (long)rec.size();
}
/* size of one written PSIO entry, -1 if absent; copy it into out (may be NULL) */
long v2b_ref_psio_entry(int unit, const char *key, char *out) {
    auto it = psi::psio_store().find({unit, key});
    if (it == psi::psio_store().end()) return -1;
    if (out) std::memcpy(out, it->second.data(), it->second.size());
    return (long)it->second.size();
}
int v2b_ref_pack_spatial(void *p, const double *x, double *d2, double *d1) {
    try {
        static_cast<RefProblem *>(p)->pack(x, d2, d1);
        return 0;
    } catch (const std::exception &e) { g_last_error = e.what(); return 1; }
}

}  // extern "C"
