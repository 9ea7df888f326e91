// Host-side code model: params reader, APM construction, row bases, ETS tables.
#include "code_model.hpp"

#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <sys/stat.h>

namespace jbp {

namespace {

long long mod_norm(long long x, long long m) {
    long long r = x % m;
    return r < 0 ? r + m : r;
}

// Extended Euclid for the modular inverse used by the Hz blocks (jointbp_ets.cpp:68-87).
bool mod_inverse(long long a, long long m, long long &inv) {
    a = mod_norm(a, m);
    if (m == 1) { inv = 0; return true; }
    long long r0 = m, r1 = a, t0 = 0, t1 = 1;
    while (r1 != 0) {
        long long q = r0 / r1;
        long long r2 = r0 - q * r1; r0 = r1; r1 = r2;
        long long t2 = t0 - q * t1; t0 = t1; t1 = t2;
    }
    if (r0 != 1) return false;
    inv = mod_norm(t0, m);
    return true;
}

int wrap(int x, int m) { int r = x % m; return r < 0 ? r + m : r; }

void finish_side(SideGraph &g, int n) {
    g.edges = g.chk_off.empty() ? 0 : g.chk_off.back();
    std::vector<int> deg(n, 0);
    for (int e = 0; e < g.edges; ++e) deg[g.chk_var[e]]++;
    g.var_off.assign(n + 1, 0);
    for (int v = 0; v < n; ++v) g.var_off[v + 1] = g.var_off[v] + deg[v];
    g.var_edge.assign(g.edges, 0);
    std::vector<int> fill(n, 0);
    for (int c = 0; c < g.m; ++c)
        for (int e = g.chk_off[c]; e < g.chk_off[c + 1]; ++e) {
            int v = g.chk_var[e];
            g.var_edge[g.var_off[v] + fill[v]++] = e;
        }
    g.dc_max = 0;
    for (int c = 0; c < g.m; ++c) g.dc_max = std::max(g.dc_max, g.chk_off[c + 1] - g.chk_off[c]);
    g.dv_max = 0;
    for (int v = 0; v < n; ++v) g.dv_max = std::max(g.dv_max, deg[v]);
    g.checks_regular = true;
    for (int c = 0; c < g.m && g.checks_regular; ++c) g.checks_regular = (g.chk_off[c + 1] - g.chk_off[c]) == g.dc_max;
    g.regular = g.checks_regular;
    for (int v = 0; v < n && g.regular; ++v) g.regular = deg[v] == g.dv_max;
}

// Row basis as build_row_basis (jointbp_ets.cpp:845-885): each check row is reduced at
// its highest set bit against the rows kept so far and kept if it survives.
void build_basis(const SideGraph &g, int n, RowBasis &b) {
    b.words = (n + 63) / 64;
    b.rank = 0;
    b.rows.clear();
    b.pivot.clear();
    b.pivot_row.assign(n, -1);
    std::vector<uint64_t> row(b.words);
    for (int c = 0; c < g.m; ++c) {
        std::fill(row.begin(), row.end(), 0);
        for (int e = g.chk_off[c]; e < g.chk_off[c + 1]; ++e) row[g.chk_var[e] >> 6] |= 1ull << (g.chk_var[e] & 63);
        for (;;) {
            int hb = -1;
            for (int w = b.words - 1; w >= 0; --w)
                if (row[w]) { hb = w * 64 + 63 - __builtin_clzll(row[w]); break; }
            if (hb < 0) break;
            int r = b.pivot_row[hb];
            if (r < 0) {
                b.pivot_row[hb] = b.rank++;
                b.pivot.push_back(hb);
                b.rows.insert(b.rows.end(), row.begin(), row.end());
                break;
            }
            const uint64_t *base = &b.rows[static_cast<size_t>(r) * b.words];
            for (int w = 0; w < b.words; ++w) row[w] ^= base[w];
        }
    }
}

std::string trim(const std::string &s) {
    size_t a = 0, e = s.size();
    while (a < e && std::isspace(static_cast<unsigned char>(s[a]))) ++a;
    while (e > a && std::isspace(static_cast<unsigned char>(s[e - 1]))) --e;
    return s.substr(a, e - a);
}

// Comma split keeping inner empty fields and dropping an empty tail.
std::vector<std::string> csv_fields(const std::string &s) {
    std::vector<std::string> out;
    std::string cur;
    for (char ch : s) {
        if (ch == ',') { out.push_back(trim(cur)); cur.clear(); }
        else cur.push_back(ch);
    }
    if (!cur.empty()) out.push_back(trim(cur));
    return out;
}

// "<K><block>:<index>" -> block * P + index.
bool parse_block_token(const std::string &tok, char kind, int P, int &id) {
    if (tok.size() < 3 || std::toupper(static_cast<unsigned char>(tok[0])) != kind) return false;
    size_t colon = tok.find(':');
    if (colon == std::string::npos) return false;
    const char *s1 = tok.c_str() + 1;
    char *end = nullptr;
    long blk = std::strtol(s1, &end, 10);
    if (end == s1) return false;
    const char *s2 = tok.c_str() + colon + 1;
    long idx = std::strtol(s2, &end, 10);
    if (end == s2) return false;
    id = static_cast<int>(blk * P + idx);
    return true;
}

bool file_size(const std::string &p, long long &sz) {
    struct stat st;
    if (stat(p.c_str(), &st) != 0) return false;
    sz = st.st_size;
    return true;
}

}  // namespace

std::string params_ets_dir(const std::string &params_path) {
    size_t slash = params_path.find_last_of('/');
    std::string dir = slash == std::string::npos ? "" : params_path.substr(0, slash + 1);
    std::string base = slash == std::string::npos ? params_path : params_path.substr(slash + 1);
    size_t dot = base.find_last_of('.');
    if (dot != std::string::npos) base = base.substr(0, dot);
    return dir + base;
}

// Params format (read_params, jointbp_ets.cpp:162-180): "P J L / seed / a[L/2] / b / c / d".
// Hx block (r, col): y = a x + b with (a, b) = (a_i, b_i) on the left half and (c_i, d_i)
// on the right half, i = (col' - r) mod L/2.  Hz block: the inverse maps of the opposite
// half at index -(col' - r) mod L/2 (build_block_matrix_hz, 126-160).  A block whose
// multiplier has no inverse mod P is rejected (the reference would index err[-1]).
std::string CodeModel::build_from_params(const std::string &path) {
    std::ifstream in(path);
    if (!in) return "cannot open params file " + path;
    long long Pl = 0;
    int J = 0, L = 0;
    unsigned long long seed = 0;
    if (!(in >> Pl >> J >> L) || !(in >> seed)) return "malformed params header in " + path;
    if (Pl <= 0 || J <= 0 || L <= 0 || L % 2 != 0) return "invalid P/J/L in " + path;
    if (Pl * L > (1LL << 28)) return "code too large";
    int L2 = L / 2;
    std::vector<long long> a(L2), b(L2), c(L2), d(L2);
    for (auto *vec : {&a, &b, &c, &d})
        for (int i = 0; i < L2; ++i)
            if (!(in >> (*vec)[i])) return "malformed params coefficients in " + path;
    P = static_cast<int>(Pl);
    n = L * P;
    int m = J * P;
    for (int s = 0; s < 2; ++s) {
        SideGraph &g = side[s];
        g.m = m;
        g.chk_off.resize(m + 1);
        for (int ch = 0; ch <= m; ++ch) g.chk_off[ch] = ch * L;
        g.chk_var.assign(static_cast<size_t>(m) * L, 0);
        for (int r = 0; r < J; ++r) {
            for (int col = 0; col < L; ++col) {
                bool left = col < L2;
                int t = left ? col : col - L2;
                long long A, B;
                if (s == 0) {
                    int idx = wrap(t - r, L2);
                    A = mod_norm(left ? a[idx] : c[idx], Pl);
                    B = mod_norm(left ? b[idx] : d[idx], Pl);
                } else {
                    int idx = wrap(-wrap(t - r, L2), L2);
                    long long mul = left ? c[idx] : a[idx];
                    long long add = left ? d[idx] : b[idx];
                    long long inv;
                    if (!mod_inverse(mod_norm(mul, Pl), Pl, inv))
                        return "Hz block (" + std::to_string(r) + "," + std::to_string(col) +
                               ") has a non-invertible multiplier";
                    A = inv;
                    B = mod_norm(-inv * mod_norm(add, Pl), Pl);
                }
                for (int x = 0; x < P; ++x) {
                    long long y = mod_norm(A * x + B, Pl);
                    g.chk_var[static_cast<size_t>(r * P + x) * L + col] = col * P + static_cast<int>(y);
                }
            }
        }
        finish_side(g, n);
        build_basis(g, n, basis[s]);
    }
    return "";
}

std::string CodeModel::build_from_checks(int n_, const std::vector<int> &xoff, const std::vector<int> &xvar,
                                         const std::vector<int> &zoff, const std::vector<int> &zvar) {
    n = n_;
    P = 0;
    const std::vector<int> *offs[2] = {&xoff, &zoff}, *vars[2] = {&xvar, &zvar};
    for (int s = 0; s < 2; ++s) {
        SideGraph &g = side[s];
        if (offs[s]->empty() || (*offs[s])[0] != 0) return "check offsets must start at 0";
        g.m = static_cast<int>(offs[s]->size()) - 1;
        g.chk_off = *offs[s];
        for (int ch = 0; ch < g.m; ++ch)
            if (g.chk_off[ch + 1] < g.chk_off[ch]) return "check offsets must be non-decreasing";
        if (static_cast<int>(vars[s]->size()) != g.chk_off[g.m]) return "check variable list size mismatch";
        g.chk_var = *vars[s];
        for (int v : g.chk_var)
            if (v < 0 || v >= n) return "check lists a variable out of range";
        finish_side(g, n);
        build_basis(g, n, basis[s]);
    }
    return "";
}

// ETS line format (read_ets_file, jointbp_ets.cpp:3199-3258): optional "X "/"Z " side
// prefix, then "vars=V<col>:<i>,... unsat=C<row>:<i>,C<row>:<i>".  Lines for the other
// side, lines without both fields and lines whose counts do not match are skipped.
// Entries whose variables or checks fall outside the code are skipped too (the
// reference would index past its arrays).
std::string ets_read_file(const std::string &path, int P, int n, int expected_vars, char side, EtsTable &out,
                          bool *opened) {
    out = EtsTable{};
    out.var_count = expected_vars;
    if (opened) *opened = false;
    if (expected_vars <= 0 || expected_vars > 32) return "ETS size must be 1..32";
    std::ifstream in(path);
    if (!in) return "cannot open " + path;
    if (opened) *opened = true;
    std::string line;
    while (std::getline(in, line)) {
        line = trim(line);
        if (line.empty()) continue;
        char line_side = 0;
        if (line.size() >= 2 && std::strchr("XxZz", line[0]) && std::isspace(static_cast<unsigned char>(line[1]))) {
            line_side = static_cast<char>(std::toupper(static_cast<unsigned char>(line[0])));
            line = trim(line.substr(1));
        }
        if ((side == 'X' || side == 'Z') && line_side != 0 && line_side != side) continue;
        size_t pv = line.find("vars="), pu = line.find("unsat=");
        if (pv == std::string::npos || pu == std::string::npos || pu < pv + 5) continue;
        auto vt = csv_fields(trim(line.substr(pv + 5, pu - (pv + 5))));
        auto ct = csv_fields(trim(line.substr(pu + 6)));
        if (static_cast<int>(vt.size()) != expected_vars || ct.size() != 2) continue;
        std::vector<int> ids(expected_vars);
        bool ok = true;
        for (int i = 0; i < expected_vars && ok; ++i) ok = parse_block_token(vt[i], 'V', P, ids[i]) && ids[i] >= 0 && ids[i] < n;
        int c0 = 0, c1 = 0;
        ok = ok && parse_block_token(ct[0], 'C', P, c0) && parse_block_token(ct[1], 'C', P, c1) && c0 >= 0 && c1 >= 0;
        if (!ok) continue;
        std::sort(ids.begin(), ids.end());
        if (c0 > c1) std::swap(c0, c1);
        out.vars.insert(out.vars.end(), ids.begin(), ids.end());
        out.key.push_back((static_cast<uint64_t>(static_cast<uint32_t>(c0)) << 32) | static_cast<uint32_t>(c1));
    }
    return "";
}

std::string CodeModel::add_ets_group(int size, const std::string &label, const std::string &path_x,
                                     const std::string &path_z) {
    EtsGroup g;
    g.size = size;
    g.label = label;
    const std::string *paths[2] = {&path_x, &path_z};
    for (int s = 0; s < 2; ++s) {
        if (paths[s]->empty()) continue;
        long long sz = 0;
        if (!file_size(*paths[s], sz) || sz == 0) continue;  // missing or empty: not loaded
        bool opened = false;
        std::string err = ets_read_file(*paths[s], P, n, size, s == 0 ? 'X' : 'Z', g.tab[s], &opened);
        if (!err.empty() && opened) return err;
        g.loaded[s] = err.empty() && g.tab[s].count() > 0;
        if (!g.loaded[s]) g.tab[s] = EtsTable{};
    }
    // check ids must be in range for the side they index
    for (int s = 0; s < 2; ++s) {
        if (!g.loaded[s]) continue;
        for (uint64_t k : g.tab[s].key)
            if (static_cast<int>(k >> 32) >= side[s].m || static_cast<int>(k & 0xffffffffu) >= side[s].m)
                return "ETS table " + *paths[s] + " lists a check outside the code";
    }
    if (g.loaded[0] || g.loaded[1]) ets.push_back(std::move(g));
    return "";
}

// Default ETS files under a directory, in the reference load order (jointbp_ets.cpp:5317-5337).
std::string CodeModel::load_ets_dir(const std::string &dir) {
    static const int sizes[] = {6, 8, 10, 12, 14, 16, 18, 20, 22};
    for (int s : sizes) {
        std::string p = dir + "/ets_" + std::to_string(s) + "_2.txt";
        std::string err = add_ets_group(s, std::to_string(s), p, p);
        if (!err.empty()) return err;
        if (s == 8) {
            std::string p4 = dir + "/ets_8_2_path4.txt";
            err = add_ets_group(8, "8p4", p4, p4);
            if (!err.empty()) return err;
        }
    }
    return "";
}


// ------------------------------------------------------------------ start-up graph checks

namespace {

// Check of each edge of a side (edge ids are check-major: chk_off[c] .. chk_off[c+1]-1).
std::vector<int> edge_checks(const SideGraph &g) {
    std::vector<int> ec(static_cast<size_t>(g.edges));
    for (int c = 0; c < g.m; ++c)
        for (int e = g.chk_off[c]; e < g.chk_off[c + 1]; ++e) ec[e] = c;
    return ec;
}

// Pairs (X check, Z check) with an odd overlap: every variable contributes each pair of its
// X and Z checks once, so a pair's overlap is the number of times it is listed.
long long odd_overlap_pairs(const SideGraph &x, const SideGraph &z, int n) {
    const std::vector<int> ecx = edge_checks(x), ecz = edge_checks(z);
    std::vector<unsigned long long> pairs;
    for (int v = 0; v < n; ++v)
        for (int a = x.var_off[v]; a < x.var_off[v + 1]; ++a)
            for (int b = z.var_off[v]; b < z.var_off[v + 1]; ++b)
                pairs.push_back(static_cast<unsigned long long>(ecx[x.var_edge[a]]) << 32 |
                                static_cast<unsigned>(ecz[z.var_edge[b]]));
    std::sort(pairs.begin(), pairs.end());
    long long odd = 0;
    for (size_t i = 0; i < pairs.size();) {
        size_t j = i;
        while (j < pairs.size() && pairs[j] == pairs[i]) ++j;
        odd += (j - i) & 1;
        i = j;
    }
    return odd;
}

// Girth of a Tanner graph (variables 0..n-1, checks n..n+m-1): breadth-first search from every
// variable; a non-tree edge between nodes at depths a and b closes a cycle of length a + b + 1
// through the start's search tree, and the shortest such cycle over all starts is the girth.
// A search stops expanding nodes at depth >= best/2, where no shorter cycle can close.
int tanner_girth(const SideGraph &g, int n) {
    const std::vector<int> ec = edge_checks(g);
    const int total = n + g.m;
    std::vector<int> depth(total), parent(total), mark(total, -1), queue(total);
    int best = 0x7fffffff;
    for (int s = 0; s < n && best > 4; ++s) {
        int head = 0, tail = 0;
        queue[tail++] = s;
        mark[s] = s;
        depth[s] = 0;
        parent[s] = -1;
        while (head < tail) {
            const int u = queue[head++];
            if (2 * depth[u] >= best) continue;
            auto visit = [&](int w) {
                if (mark[w] != s) {
                    mark[w] = s;
                    depth[w] = depth[u] + 1;
                    parent[w] = u;
                    queue[tail++] = w;
                } else if (w != parent[u]) {
                    best = std::min(best, depth[u] + depth[w] + 1);
                }
            };
            if (u < n) {
                for (int k = g.var_off[u]; k < g.var_off[u + 1]; ++k) visit(n + ec[g.var_edge[k]]);
            } else {
                const int c = u - n;
                for (int e = g.chk_off[c]; e < g.chk_off[c + 1]; ++e) visit(g.chk_var[e]);
            }
        }
    }
    return best == 0x7fffffff ? 0 : best;
}

}  // namespace

GraphChecks graph_checks(const CodeModel &m) {
    GraphChecks r;
    r.odd_pairs = odd_overlap_pairs(m.side[0], m.side[1], m.n);
    r.girth[0] = tanner_girth(m.side[0], m.n);
    r.girth[1] = tanner_girth(m.side[1], m.n);
    return r;
}

}  // namespace jbp
