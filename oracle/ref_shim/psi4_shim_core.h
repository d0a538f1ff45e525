/*
 * Test-only stand-ins for the handful of Psi4 declarations that hilbert's
 * v2RDM constraint-map sources include.  These are NOT Psi4: they are the
 * minimum surface (names, member variables, trivial containers) needed to
 * compile hilbert's own basis.cc / d2.cc / spin.cc / q2.cc / g2.cc / t*.cc /
 * tei.cc against plain C++ so that those files can serve as the bit-exact
 * oracle for the B200 maps.  Nothing here is used by the product library.
 */
#ifndef V2B_PSI4_SHIM_CORE_H
#define V2B_PSI4_SHIM_CORE_H

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#ifndef PSI_API
#define PSI_API
#endif

/* packed lower-triangle index used by hilbert for symmetric (ij|kl) storage */
#ifndef INDEX
#define INDEX(i, j) ((i) > (j) ? ((long)(i) * ((long)(i) + 1) / 2 + (long)(j)) \
                               : ((long)(j) * ((long)(j) + 1) / 2 + (long)(i)))
#endif

namespace psi {

class PsiException : public std::runtime_error {
  public:
    PsiException(const std::string &msg, const char *file, int line)
        : std::runtime_error(msg + " (" + file + ":" + std::to_string(line) + ")") {}
};

/* output stream: the oracle is silent unless V2B_REF_VERBOSE is set */
class PsiOutStream {
  public:
    template <typename... Args>
    void Printf(const char *fmt, Args... args) {
        if (std::getenv("V2B_REF_VERBOSE")) std::printf(fmt, args...);
    }
    void Printf(const char *fmt) {
        if (std::getenv("V2B_REF_VERBOSE")) std::printf("%s", fmt);
    }
};
extern std::shared_ptr<PsiOutStream> outfile;

class Dimension {
  public:
    Dimension() {}
    explicit Dimension(int n, const std::string & = "") : v_(n, 0) {}
    int &operator[](int h) { return v_[h]; }
    const int &operator[](int h) const { return v_[h]; }
    int n() const { return (int)v_.size(); }
    int sum() const { int s = 0; for (int x : v_) s += x; return s; }
  private:
    std::vector<int> v_;
};

class Vector {
  public:
    Vector() {}
    Vector(const std::string &, long n) : blocks_(1, std::vector<double>(n, 0.0)) {}
    explicit Vector(long n) : blocks_(1, std::vector<double>(n, 0.0)) {}
    explicit Vector(const Dimension &d) {
        for (int h = 0; h < d.n(); h++) blocks_.push_back(std::vector<double>(d[h] > 0 ? d[h] : 1, 0.0));
    }
    double *pointer(int h = 0) { return blocks_[h].data(); }
    void zero() { for (auto &b : blocks_) std::fill(b.begin(), b.end(), 0.0); }
    long dim(int h = 0) const { return (long)blocks_[h].size(); }
  private:
    std::vector<std::vector<double>> blocks_;
};
typedef std::shared_ptr<Vector> SharedVector;

class Matrix {
  public:
    Matrix() {}
    Matrix(int r, int c) { alloc(r, c); }
    Matrix(const std::string &, int r, int c) { alloc(r, c); }
    double **pointer(int h = 0) { (void)h; return rows_.data(); }
    void zero() { std::fill(data_.begin(), data_.end(), 0.0); }
  private:
    void alloc(int r, int c) {
        data_.assign((size_t)r * c + 1, 0.0);
        rows_.resize(r > 0 ? r : 1);
        for (int i = 0; i < r; i++) rows_[i] = data_.data() + (size_t)i * c;
    }
    std::vector<double> data_;
    std::vector<double *> rows_;
};
typedef std::shared_ptr<Matrix> SharedMatrix;

/* option store: only the accessors hilbert's map-side code calls */
class Options {
  public:
    struct Data {
        bool changed = false;
        bool has_changed() const { return changed; }
    };
    std::string get_str(const std::string &k) { return s_.count(k) ? s_[k] : std::string(); }
    bool get_bool(const std::string &k) { return b_.count(k) ? b_[k] : false; }
    int get_int(const std::string &k) { return i_.count(k) ? i_[k] : 0; }
    double get_double(const std::string &k) { return d_.count(k) ? d_[k] : 0.0; }
    Data &operator[](const std::string &k) { return data_[k]; }
    void set_str(const std::string &k, const std::string &v) { s_[k] = v; }
    void set_bool(const std::string &k, bool v) { b_[k] = v; }
    void set_int(const std::string &k, int v) { i_[k] = v; }
    void set_double(const std::string &k, double v) { d_[k] = v; }
  private:
    std::map<std::string, std::string> s_;
    std::map<std::string, bool> b_;
    std::map<std::string, int> i_;
    std::map<std::string, double> d_;
    std::map<std::string, Data> data_;
};

class Molecule {};
class BasisSet { public: int nbf() const { return 0; } };

/* Wavefunction: just the data members the compiled hilbert files touch */
class Wavefunction {
  public:
    explicit Wavefunction(Options &options) : options_(options) {}
    virtual ~Wavefunction() {}
    virtual double compute_energy() = 0;
    virtual bool same_a_b_orbs() const { return same_a_b_orbs_; }
    virtual bool same_a_b_dens() const { return same_a_b_dens_; }
  protected:
    Options &options_;
    std::shared_ptr<Wavefunction> reference_wavefunction_;
    std::shared_ptr<Molecule> molecule_;
    int nirrep_ = 1;
    int nmo_ = 0;
    int nso_ = 0;
    int nalpha_ = 0;   // Psi4's Wavefunction members; v2RDMSolver declares its own
    int nbeta_ = 0;
    long memory_ = 0;
    double energy_ = 0.0;
    double efzc_ = 0.0;
    bool same_a_b_orbs_ = false;
    bool same_a_b_dens_ = false;
    std::string name_;
    Dimension nalphapi_, nbetapi_, frzcpi_, frzvpi_, nmopi_, nsopi_;
    std::shared_ptr<Vector> epsilon_a_, epsilon_b_;
    SharedMatrix Ca_, Cb_, Fa_, Fb_, Da_, Db_, S_, AO2SO_, Lagrangian_, gradient_;
};
typedef std::shared_ptr<Wavefunction> SharedWavefunction;

struct iwlbuf { int dummy; };

/* LAPACK's dsyevd with Psi4's libqt calling convention (the matrix as
 * LAPACK sees it: eigenvectors come back as contiguous columns); defined by
 * the focas harness, which links LAPACK */
int C_DSYEVD(char jobz, char uplo, int n, double *a, int lda, double *w, double *work, int lwork,
             int *iwork, int liwork);

/* BLAS level-1 helpers used by the maps (plain loops: no FMA contraction) */
inline void C_DCOPY(size_t n, double *x, int incx, double *y, int incy) {
    for (size_t i = 0; i < n; i++) y[i * incy] = x[i * incx];
}
inline void C_DAXPY(size_t n, double a, double *x, int incx, double *y, int incy) {
    for (size_t i = 0; i < n; i++) y[i * incy] += a * x[i * incx];
}
inline double C_DDOT(size_t n, double *x, int incx, double *y, int incy) {
    double s = 0.0;
    for (size_t i = 0; i < n; i++) s += x[i * incx] * y[i * incy];
    return s;
}
inline double C_DNRM2(size_t n, double *x, int incx) {
    double s = 0.0;
    for (size_t i = 0; i < n; i++) s += x[i * incx] * x[i * incx];
    return std::sqrt(s);
}
inline void C_DSCAL(size_t n, double a, double *x, int incx) {
    for (size_t i = 0; i < n; i++) x[i * incx] *= a;
}

/* PSIO: files are kept in memory, one byte string per (unit, entry), so the
   oracle can read back what the reference's writers emit.  The store is
   process-wide (psio_store()); open(PSIO_OPEN_NEW) empties the unit. */
struct psio_address {
    size_t page = 0, offset = 0;
};
static const psio_address PSIO_ZERO = {0, 0};
enum { PSIO_OPEN_NEW = 0, PSIO_OPEN_OLD = 1 };
typedef std::map<std::pair<int, std::string>, std::string> PsioStore;
inline PsioStore &psio_store() {
    static PsioStore store;
    return store;
}
class PSIO {
  public:
    void open(int unit, int mode) {
        if (mode != PSIO_OPEN_NEW) return;
        PsioStore &s = psio_store();
        for (auto it = s.begin(); it != s.end();)
            it = it->first.first == unit ? s.erase(it) : std::next(it);
    }
    void close(int, int) {}
    bool exists(int unit) {
        for (auto &kv : psio_store())
            if (kv.first.first == unit) return true;
        return false;
    }
    void write(int unit, const char *key, char *buf, size_t size, psio_address start, psio_address *end) {
        std::string &e = psio_store()[{unit, key}];
        if (e.size() < start.offset + size) e.resize(start.offset + size);
        std::memcpy(&e[start.offset], buf, size);
        if (end) *end = psio_address{0, start.offset + size};
    }
    void write_entry(int unit, const char *key, char *buf, size_t size) {
        write(unit, key, buf, size, PSIO_ZERO, nullptr);
    }
    void read(int unit, const char *key, char *buf, size_t size, psio_address start, psio_address *end) {
        const std::string &e = psio_store().at({unit, key});
        std::memcpy(buf, e.data() + start.offset, size);
        if (end) *end = psio_address{0, start.offset + size};
    }
    void read_entry(int unit, const char *key, char *buf, size_t size) { read(unit, key, buf, size, PSIO_ZERO, nullptr); }
};

/* IWL: every write_value call is recorded, per unit, in call order, with the
   cutoff the file was opened with; the harness reads the records back.
   Psi4's own buffers and its cutoff test are not restated here. */
struct IwlRecord {
    int p, q, r, s;
    double value;
};
struct IwlFile {
    double cutoff = 0.0;
    std::vector<IwlRecord> records;
};
inline std::map<int, IwlFile> &iwl_store() {
    static std::map<int, IwlFile> store;
    return store;
}
class IWL {
  public:
    IWL(PSIO *, int unit, double cutoff, int, int) : unit_(unit) {
        iwl_store()[unit] = IwlFile();
        iwl_store()[unit].cutoff = cutoff;
    }
    void write_value(int p, int q, int r, int s, double value, int, const std::string &, int) {
        iwl_store()[unit_].records.push_back(IwlRecord{p, q, r, s, value});
    }
    void flush(int) {}
    void set_keep_flag(int) {}
    void close() {}
  private:
    int unit_;
};

}  // namespace psi

/* stand-in unit numbers for the MO-basis 2-RDM files the IWL writer opens */
#ifndef PSIF_MO_AA_TPDM
#define PSIF_MO_AA_TPDM 9001
#define PSIF_MO_AB_TPDM 9002
#define PSIF_MO_BB_TPDM 9003
#endif

#endif
