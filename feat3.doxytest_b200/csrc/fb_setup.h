// Host-side set-up of the multigrid hierarchy: validation, explicit-zero removal on the transfer
// matrices, reverse Cuthill-McKee reordering, index narrowing to u32, inverse diagonals and the
// exact coarse-grid inverse.  Plain C++ (no CUDA), run once per solver.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace fb
{
  struct HostCsr
  {
    uint32_t rows = 0, cols = 0;
    std::vector<uint32_t> rp, col;
    std::vector<double> val;
    uint64_t nnz() const { return col.size(); }
  };

  struct HostLevel
  {
    HostCsr A, P, R;            // P: this <- coarser, R: coarser <- this (empty on the coarsest)
    std::vector<uint8_t> dmask; // 1 = Dirichlet DOF
    std::vector<uint64_t> fidx; // Dirichlet DOFs (caller numbering)
    std::vector<double> fval;
    std::vector<uint32_t> perm; // device row k = caller row perm[k] (empty = identity)
    bool set = false;
  };

  // Converts a caller CSR (u64) into a HostCsr; drop_zeros removes stored entries equal to +-0.
  // Returns an empty string on success, else a message.
  std::string import_csr(HostCsr& out, uint64_t rows, uint64_t cols, uint64_t nnz, const uint64_t* rp,
                         const uint64_t* col, const double* val, bool drop_zeros);

  // Reverse Cuthill-McKee ordering of the symmetric pattern of A: perm[k] = old row.
  std::vector<uint32_t> rcm_order(const HostCsr& A);

  // B = Pr * M * Pc^T with row order perm_r (new row k = old row perm_r[k]) and column map
  // inv_c (new column = inv_c[old column]); entries keep their stored order within each row.
  HostCsr permute(const HostCsr& M, const std::vector<uint32_t>& perm_r, const std::vector<uint32_t>& inv_c);

  // omega / a_ii, a_ii = 0 when the row stores no diagonal entry (JacobiPrecond::init_numeric).
  std::vector<double> inv_diagonal(const HostCsr& A, double omega);

  // Inverse of A restricted to the non-Dirichlet DOFs (Gauss-Jordan, partial pivoting), row-major
  // m x m, and the free DOF list.
  void coarse_inverse(const HostCsr& A, const std::vector<uint8_t>& dmask, std::vector<uint32_t>& free_dofs,
                      std::vector<double>& inv);

  std::vector<uint32_t> inverse_perm(const std::vector<uint32_t>& perm);

  // Order of a triangular sweep (SOR / SSOR): the rows of colour c are order[cofs[c] .. cofs[c+1]),
  // colours processed in ascending order, rows of one colour independent of each other.
  struct SweepOrder
  {
    std::vector<uint32_t> order, cofs;
    uint32_t colours() const { return uint32_t(cofs.size()) - 1u; }
  };
  // Dependency levels of the sequential sweep over the entries left of the diagonal (forward) or
  // right of it (backward): a row's level is one more than the highest level among the rows its
  // entries couple it to on that side.  Sweeping level after level gives every row the same inputs
  // as the sequential sweep, so the result is identical.
  SweepOrder sweep_levels(const HostCsr& A, bool backward);
  // Greedy colouring of the symmetric pattern (rows in ascending order take the smallest colour no
  // coupled, already coloured row has), colours ordered by ascending row count, ties by number:
  // the colouring of the coloured sweeps.
  SweepOrder greedy_colours(const HostCsr& A);

  // A matrix in the device layout of the solvers: sliced ELL with 32-row slices (entry k of row
  // 32s+lane at soff[s] + 32k + lane, stored order kept), or plain ELL (uniform width kw, when it
  // stores at most 12.5% more entries).  Rows flagged in `empty` are stored without entries;
  // padding has value 0 and the zero-slot column `cols` (or offset 0 for narrow storage).  Square
  // matrices whose |col - row| fits in int16 get 2-byte column offsets (dcol) instead of col.
  // Diagonal storage (allow_diag, square matrices): when every stored entry lies on one of at most
  // DIAG_MAX diagonals and every row's columns are strictly increasing, the matrix is stored as
  // plain ELL whose entry k of every row is the diagonal doff[k] (column = row + doff[k]), without
  // column indices: a row's entries keep their stored order, the diagonals it lacks hold value 0
  // (at most 12.5% padding, except for matrices of at most DIAG_SMALL_ROWS rows).
  constexpr uint32_t DIAG_MAX = 27;
  constexpr uint32_t DIAG_SMALL_ROWS = 4096;   // up to this many rows: no padding limit
  struct HostSell
  {
    uint32_t rows = 0, cols = 0, kw = 0;
    uint64_t nnz = 0, entries = 0;
    bool narrow = false;
    std::vector<uint32_t> soff;
    std::vector<uint32_t> col;
    std::vector<int16_t> dcol;
    std::vector<int32_t> doff;   // diagonal storage: the offsets, ascending; empty otherwise
    std::vector<double> val;
    // slot of entry j (column c) of row r, stored order within the row
    uint64_t slot(uint32_t r, uint32_t j, uint32_t c) const;
  };
  HostSell build_sell(const HostCsr& M, const std::vector<uint8_t>* empty, bool allow_narrow = true,
                      bool allow_diag = false);
} // namespace fb

// the opaque hierarchy handle of the C ABI: levels finest first, as pushed by the caller
struct fb_hierarchy
{
  std::vector<fb::HostLevel> levels;
};
