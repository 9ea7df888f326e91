// Host-side model of a CSS code for the joint X/Z BP decoder.
//
// Builds the X/Z check lists from the reference params-file format (APM construction,
// jointbp_ets.cpp:36-180 and 628-648), the per-variable edge lists in ascending check
// order (build_var_adjacency, 922-935), the GF(2) row bases used for the
// stabilizer-equivalence test (build_row_basis, 845-885) and the ETS tables
// (read_ets_file, 3199-3258).  Everything here runs once at start-up.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace jbp {

struct SideGraph {
    int m = 0;                    // checks
    int edges = 0;
    std::vector<int> chk_off;     // m+1; edge id = chk_off[c] + position (check-major)
    std::vector<int> chk_var;     // variable of each edge
    std::vector<int> var_off;     // n+1
    std::vector<int> var_edge;    // edges of each variable, ascending check index
    int dc_max = 0, dv_max = 0;
    bool regular = false;         // every check has dc_max edges and every variable dv_max
    bool checks_regular = false;  // every check has dc_max edges (variables may have fewer than dv_max)
};

// GF(2) basis of a check matrix's row space: rows reduced at their highest bit.
struct RowBasis {
    int words = 0;
    int rank = 0;
    std::vector<uint64_t> rows;   // rank * words
    std::vector<int> pivot;       // highest bit of each row
    std::vector<int> pivot_row;   // n entries: basis row whose pivot is that column, or -1
};

// ETS table of one size and one side; entries keep file order.
struct EtsTable {
    int var_count = 0;
    std::vector<int> vars;        // count * var_count, sorted per entry
    std::vector<uint64_t> key;    // (c0 << 32) | c1, c0 < c1
    int count() const { return static_cast<int>(key.size()); }
};

struct EtsGroup {
    int size = 0;
    std::string label;
    bool loaded[2] = {false, false};
    EtsTable tab[2];
};

struct CodeModel {
    int n = 0;
    int P = 0;                    // circulant size of the APM construction (0 when built from lists)
    SideGraph side[2];            // 0 = X checks (x-bits), 1 = Z checks (z-bits)
    RowBasis basis[2];            // row space of Hx (side 0) and Hz (side 1)
    std::vector<EtsGroup> ets;    // groups in the reference order 6, 8, 8p4, 10, ..., 22

    // Returns an empty string on success, else the error.
    std::string build_from_params(const std::string &path);
    std::string build_from_checks(int n, const std::vector<int> &xoff, const std::vector<int> &xvar,
                                  const std::vector<int> &zoff, const std::vector<int> &zvar);
    // Loads the ETS groups from a directory (default file names); missing files are skipped.
    std::string load_ets_dir(const std::string &dir);
    // Loads one group from explicit files (empty path = not loaded).
    std::string add_ets_group(int size, const std::string &label, const std::string &path_x,
                              const std::string &path_z);
};

std::string ets_read_file(const std::string &path, int P, int n, int expected_vars, char side, EtsTable &out,
                          bool *opened);

// Start-up graph checks of a CSS code (the reference's check_hx_hz_orthogonality and
// compute_girth, jointbp_ets.cpp:1070-1171): the number of (X check, Z check) pairs that share
// an odd number of variables (0 for a valid CSS code), and the girth of each side's Tanner
// graph (0 when it has no cycle).
struct GraphChecks {
    long long odd_pairs = 0;
    int girth[2] = {0, 0};
};
GraphChecks graph_checks(const CodeModel &m);
std::string params_ets_dir(const std::string &params_path);

}  // namespace jbp
