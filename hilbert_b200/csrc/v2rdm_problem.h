// Host-side description of one C1 v2RDM boundary-point problem: geminal
// tables, primal block layout, b, c, guesses, and the constraint operator A
// emitted as packed sparse rows (A) and packed sparse columns (A^T).
//
// Layout and ordering follow hilbert's v2RDMSolver:
//   tables         src/v2rdm_casscf/basis.cc:426-533
//   primal blocks  src/v2rdm_casscf/v2rdm_solver.cc:3729-4079 (set_primal_offsets)
//   dual rows      src/v2rdm_casscf/v2rdm_solver.cc:2995-3050 (bpsdp_Au call order)
//   b              src/v2rdm_casscf/v2rdm_solver.cc:1826-2070 (BuildConstraints)
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace v2b {

enum Positivity { POS_D = 0, POS_DQ = 1, POS_DG = 2, POS_DQG = 3, POS_DQGT2 = 4, POS_DQGT1 = 5,
                  POS_DQGT1T2 = 6 };

struct ProblemSpec {
    int nmo = 0;          // active orbitals (C1, no frozen/restricted orbitals)
    int nalpha = 0;
    int nbeta = 0;
    int positivity = POS_DQG;
    bool constrain_spin = true;
    bool constrain_sz = true;
    bool hubbard_multiplicity = false;  // 2*(na-nb)+1 (Hubbard) vs (na-nb)+1 (external)
    bool constrain_d3 = false;          // CONSTRAIN_D3 (v2rdm_solver.cc:4120-4122)
    bool constrain_q3 = false;          // CONSTRAIN_Q3, implies D3 (:4132-4135)
    bool constrain_e3 = false;          // CONSTRAIN_E3, implies D3 (:4124-4127)
    bool constrain_f3 = false;          // CONSTRAIN_F3, implies D3 (:4128-4131)
    bool constrain_d4 = false;          // CONSTRAIN_D4, implies D3 (:4144-4149)
    bool doci = false;                  // the v2RDM-DOCI program (src/v2rdm_doci)
    int batch_parts = 0;                // > 0: independent problems along the diagonal
};

// offsets of the v2RDM-DOCI primal blocks (v2rdm_doci_solver.cc:542-600)
struct DociOffsets {
    int64_t d2s2 = -1, d2s0 = -1, d1 = -1, q2s2 = -1, q2s0 = -1, g2s2 = -1, g2s0 = -1;
    int64_t d3s3 = -1, d3s1 = -1, t1aaa = -1, t1aab = -1, t1s1 = -1, t2s1 = -1, t2 = -1;
};

// Packed sparse operator: entry = col (bits 0..26) | coef code (27..30) | group flag (31).
// Within a row the entries are stored in the order the reference accumulates them.
struct PackedOperator {
    int64_t nrows = 0;
    int64_t ncols = 0;
    std::vector<uint32_t> row_ptr;   // nrows + 1 (host check: nnz < 2^32)
    std::vector<uint32_t> entries;
    std::vector<double> palette;     // <= 16 distinct coefficients
};

constexpr uint32_t kColBits = 27;
constexpr uint32_t kColMask = (1u << kColBits) - 1u;
constexpr uint32_t kGroupFlag = 1u << 31;

struct Problem {
    ProblemSpec spec;
    int n = 0, gab = 0, gaa = 0, mult = 1;
    bool q2 = false, g2 = false, t1 = false, t2 = false, d3 = false, q3 = false, e3 = false, f3 = false;
    bool d4 = false;
    std::vector<int> bas_ab, ibas_ab, bas_aa, ibas_aa;
    // triplets (basis.cc:640-727, C1): aba = every (i, j, k), numbered
    // i n^2 + j n + k; aab = those with i < j, in the same order
    int trip_aaa = 0, trip_aab = 0, trip_aba = 0;
    std::vector<int> bas_aaa;        // 3 per aaa triplet (i < j < k)
    std::vector<int> bas_aab;        // 3 per aab triplet
    // triplet numbers of (a, b, c) at a n^2 + b n + c: aaa for any order of
    // the set, aab for either order of the alpha pair (a, b); -999 otherwise
    std::vector<int> ibas_aaa, ibas_aab;
    int64_t t1aaa = -1, t1bbb = -1, t1aab = -1, t1bba = -1;
    int64_t t2aaa = -1, t2bbb = -1, t2aab = -1, t2bba = -1;
    int64_t d3aaa = -1, d3bbb = -1, d3aab = -1, d3bba = -1;
    int64_t q3aaa = -1, q3bbb = -1, q3aab = -1, q3bba = -1;
    int64_t e3aaa = -1, e3bbb = -1, e3aab = -1, e3bba = -1;
    int64_t f3aaa = -1, f3bbb = -1, f3aab = -1, f3bba = -1;
    int64_t d4aaaa = -1, d4aaab = -1, d4aabb = -1, d4bbba = -1, d4bbbb = -1;
    // quartets (basis.cc:747-900): aaaa i<j<k<l, aaab i<j<k with any l, aabb
    // i<j with k<l; numbers at ((a n + b) n + c) n + d for every order the
    // reference maps to the same quartet, -999 otherwise
    int quad_aaaa = 0, quad_aaab = 0, quad_aabb = 0;
    std::vector<int> ibas_aaaa, ibas_aaab, ibas_aabb;
    int64_t d2ab = -1, d2aa = -1, d2bb = -1, d200 = -1, d1a = -1, d1b = -1, q1a = -1, q1b = -1;
    int64_t q2ab = -1, q2aa = -1, q2bb = -1, g2ab = -1, g2ba = -1, g2aa = -1;
    DociOffsets doci;                // spec.doci only
    int64_t n_primal = 0, n_dual = 0;
    std::vector<int> dims;           // PSD block sizes, in primal order
    std::vector<int64_t> block_off;  // offset of each block in x

    int iab(int i, int j) const { return ibas_ab[i * n + j]; }
    int iaa(int i, int j) const { return ibas_aa[i * n + j]; }
};

// Throws std::invalid_argument on bad sizes.
Problem make_problem(const ProblemSpec &spec);

void build_b(const Problem &p, double *b);
// 1D periodic Hubbard ring: h_{i,i+-1 mod n} = -t, (ii|ii) = U
void build_c_hubbard(const Problem &p, double t, double U, double *c);
// external Hamiltonian: h[i*n+j], g[i*n^3+j*n^2+k*n+l] = (ij|kl)
void build_c_external(const Problem &p, const double *h, const double *g, double *c);
void guess_random(const Problem &p, double *x);
void guess_hf(const Problem &p, double *x);   // v2RDM only (DOCI's guess is the random one)

PackedOperator build_A(const Problem &p);    // rows = dual constraints
PackedOperator build_AT(const Problem &p);   // rows = primal variables

// Independent problems as one: x, b, c, y concatenated in order, the PSD
// blocks concatenated, A block diagonal (each part's packed rows with its
// columns shifted and its coefficient codes mapped into one palette).
// Throws std::invalid_argument when the parts' coefficients do not fit one
// 16-entry palette or the columns 27 bits.
void make_batch(const std::vector<const Problem *> &parts, const std::vector<const PackedOperator *> &A,
                const std::vector<const PackedOperator *> &AT, Problem &out, PackedOperator &outA,
                PackedOperator &outAT);

}  // namespace v2b
