// Graph file readers: Matrix Market, METIS and DIMACS into int32 CSR.
//
// They follow the reference's readers (b40c/graph/builder/market.cuh,
// metis.cuh, dimacs.cuh) in what a file means:
//   * Matrix Market coordinate: each entry "a b [value]" is the directed edge
//     (row b-1, column a-1) (market.cuh:106-112); with `undirected` the
//     reverse edge follows it; rows are then stably sorted, so each row keeps
//     file order (csr_graph.cuh:108-152);
//   * METIS: header "n m [fmt]", then line i lists vertex i's neighbours,
//     1-based; the file already stores both directions (metis.cuh:80-130);
//   * DIMACS: "p <type> n m" and arcs "a u v w"; with `undirected` each arc is
//     preceded by its reverse (dimacs.cuh:150-175); rows are stably sorted.
// '%' (Market, METIS) and 'c' (DIMACS) lines are comments.  Unlike the
// reference, malformed input is rejected with a message instead of printing
// and returning -1, and a directed file whose rows are out of order is still
// sorted into a valid CSR.  Edge weights are read past and dropped.

#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "b40c_bfs.h"
#include "host_common.h"

using namespace b40c_b200;

namespace {

struct File {
    FILE *f = nullptr;
    explicit File(const char *path) : f(path ? fopen(path, "r") : nullptr) {}
    ~File() {
        if (f) fclose(f);
    }
};

// Reads one line (any length) into buf; false at end of file.
bool read_line(FILE *f, std::vector<char> &buf) {
    buf.clear();
    int c;
    while ((c = fgetc(f)) != EOF) {
        if (c == '\n') break;
        buf.push_back(char(c));
    }
    if (c == EOF && buf.empty()) return false;
    buf.push_back('\0');
    return true;
}

bool blank(const char *s) {
    for (; *s; s++)
        if (*s != ' ' && *s != '\t' && *s != '\r') return false;
    return true;
}

// Stable CSR of (rows[k], cols[k]) in list order.
int coo_to_csr(long long nodes, const std::vector<int> &rows, const std::vector<int> &cols, b40c_csr_t *out) {
    return b40c_graph_from_coo(int(nodes), int64_t(rows.size()), rows.data(), cols.data(), out);
}

}  // namespace

extern "C" int b40c_graph_read_market(const char *path, int undirected, b40c_csr_t *out) {
    if (!path || !out) return set_error(B40C_ERR_INVALID_VALUE, "read_market: NULL argument");
    File file(path);
    if (!file.f) return set_error(B40C_ERR_INVALID_VALUE, "read_market: cannot open %s (%s)", path, strerror(errno));
    std::vector<char> line;
    long long nodes = -1, declared = -1, lineno = 0;
    std::vector<int> rows, cols;
    while (read_line(file.f, line)) {
        lineno++;
        const char *s = line.data();
        if (s[0] == '%' || blank(s)) continue;
        if (nodes < 0) {
            long long nx, ny, ne;
            if (sscanf(s, "%lld %lld %lld", &nx, &ny, &ne) != 3)
                return set_error(B40C_ERR_INVALID_VALUE, "read_market: %s:%lld: invalid problem description", path,
                                 lineno);
            if (nx != ny)
                return set_error(B40C_ERR_INVALID_VALUE, "read_market: %s: not square (%lld, %lld)", path, nx, ny);
            if (nx <= 0 || nx > INT32_MAX - 1 || ne < 0 || (undirected ? 2 * ne : ne) > INT32_MAX - 8)
                return set_error(B40C_ERR_INVALID_VALUE, "read_market: %s: sizes out of range", path);
            nodes = nx;
            declared = ne;
            rows.reserve(size_t(undirected ? 2 * ne : ne));
            cols.reserve(rows.capacity());
            continue;
        }
        long long a, b;
        if (sscanf(s, "%lld %lld", &a, &b) != 2)
            return set_error(B40C_ERR_INVALID_VALUE, "read_market: %s:%lld: badly formed edge", path, lineno);
        if (a < 1 || b < 1 || a > nodes || b > nodes)
            return set_error(B40C_ERR_INVALID_VALUE, "read_market: %s:%lld: vertex out of range", path, lineno);
        if ((long long)(undirected ? rows.size() / 2 : rows.size()) >= declared)
            return set_error(B40C_ERR_INVALID_VALUE, "read_market: %s: more than %lld edges", path, declared);
        rows.push_back(int(b - 1));
        cols.push_back(int(a - 1));
        if (undirected) {
            rows.push_back(int(a - 1));
            cols.push_back(int(b - 1));
        }
    }
    if (nodes < 0) return set_error(B40C_ERR_INVALID_VALUE, "read_market: %s: no graph found", path);
    if ((long long)(undirected ? rows.size() / 2 : rows.size()) != declared)
        return set_error(B40C_ERR_INVALID_VALUE, "read_market: %s: only %zu of %lld edges read", path,
                         undirected ? rows.size() / 2 : rows.size(), declared);
    return coo_to_csr(nodes, rows, cols, out);
}

extern "C" int b40c_graph_read_metis(const char *path, b40c_csr_t *out) {
    if (!path || !out) return set_error(B40C_ERR_INVALID_VALUE, "read_metis: NULL argument");
    File file(path);
    if (!file.f) return set_error(B40C_ERR_INVALID_VALUE, "read_metis: cannot open %s (%s)", path, strerror(errno));
    std::vector<char> line;
    long long nodes = -1, m = 0, lineno = 0, v = 0;
    std::vector<int> row_offsets, cols;
    while (read_line(file.f, line)) {
        lineno++;
        const char *s = line.data();
        if (s[0] == '%') continue;
        if (nodes < 0) {
            if (blank(s)) continue;
            long long fmt = 0;
            int got = sscanf(s, "%lld %lld %lld", &nodes, &m, &fmt);
            if (got < 2 || nodes <= 0 || nodes > INT32_MAX - 1 || m < 0 || 2 * m > INT32_MAX - 8)
                return set_error(B40C_ERR_INVALID_VALUE, "read_metis: %s:%lld: invalid header", path, lineno);
            if (got == 3 && fmt % 10 != 0)
                return set_error(B40C_ERR_NOT_SUPPORTED, "read_metis: %s: weighted METIS graphs are not read", path);
            row_offsets.reserve(size_t(nodes) + 1);
            cols.reserve(size_t(2 * m));
            continue;
        }
        if (v >= nodes) {
            if (blank(s)) continue;
            return set_error(B40C_ERR_INVALID_VALUE, "read_metis: %s: more than %lld vertex lines", path, nodes);
        }
        row_offsets.push_back(int(cols.size()));
        char *p = line.data();
        for (;;) {
            char *end;
            long long x = strtoll(p, &end, 10);
            if (end == p) break;
            if (x < 1 || x > nodes)
                return set_error(B40C_ERR_INVALID_VALUE, "read_metis: %s:%lld: neighbour %lld out of range", path,
                                 lineno, x);
            if ((long long)cols.size() >= 2 * m)
                return set_error(B40C_ERR_INVALID_VALUE, "read_metis: %s: more than %lld directed edges", path,
                                 2 * m);
            cols.push_back(int(x - 1));
            p = end;
        }
        v++;
    }
    if (nodes < 0) return set_error(B40C_ERR_INVALID_VALUE, "read_metis: %s: no graph found", path);
    while ((long long)row_offsets.size() < nodes) row_offsets.push_back(int(cols.size()));
    row_offsets.push_back(int(cols.size()));
    out->nodes = nodes;
    out->edges = (int64_t)cols.size();
    out->row_offsets = (int *)malloc(sizeof(int) * row_offsets.size());
    out->column_indices = (int *)malloc(sizeof(int) * (cols.size() + 4));
    if (!out->row_offsets || !out->column_indices) {
        free(out->row_offsets);
        free(out->column_indices);
        out->row_offsets = out->column_indices = nullptr;
        return set_error(B40C_ERR_MEMORY_ALLOCATION, "read_metis: host allocation failed");
    }
    memcpy(out->row_offsets, row_offsets.data(), sizeof(int) * row_offsets.size());
    if (!cols.empty()) memcpy(out->column_indices, cols.data(), sizeof(int) * cols.size());
    memset(out->column_indices + cols.size(), 0, 4 * sizeof(int));
    return B40C_SUCCESS;
}

extern "C" int b40c_graph_read_dimacs(const char *path, int undirected, b40c_csr_t *out) {
    if (!path || !out) return set_error(B40C_ERR_INVALID_VALUE, "read_dimacs: NULL argument");
    File file(path);
    if (!file.f) return set_error(B40C_ERR_INVALID_VALUE, "read_dimacs: cannot open %s (%s)", path, strerror(errno));
    std::vector<char> line;
    long long nodes = -1, declared = 0, lineno = 0, arcs = 0;
    std::vector<int> rows, cols;
    while (read_line(file.f, line)) {
        lineno++;
        const char *s = line.data();
        if (s[0] == 'p') {
            char kind[64];
            long long n, e;
            if (sscanf(s, "p %63s %lld %lld", kind, &n, &e) != 3 || n <= 0 || n > INT32_MAX - 1 || e < 0 ||
                (undirected ? 2 * e : e) > INT32_MAX - 8)
                return set_error(B40C_ERR_INVALID_VALUE, "read_dimacs: %s:%lld: invalid problem line", path, lineno);
            nodes = n;
            declared = e;
            rows.reserve(size_t(undirected ? 2 * e : e));
            cols.reserve(rows.capacity());
        } else if (s[0] == 'a') {
            if (nodes < 0) return set_error(B40C_ERR_INVALID_VALUE, "read_dimacs: %s: arc before problem line", path);
            long long u, v;
            if (sscanf(s, "a %lld %lld", &u, &v) != 2 || u < 1 || v < 1 || u > nodes || v > nodes)
                return set_error(B40C_ERR_INVALID_VALUE, "read_dimacs: %s:%lld: bad arc", path, lineno);
            if (++arcs > declared)
                return set_error(B40C_ERR_INVALID_VALUE, "read_dimacs: %s: more than %lld arcs", path, declared);
            if (undirected) {
                rows.push_back(int(v - 1));
                cols.push_back(int(u - 1));
            }
            rows.push_back(int(u - 1));
            cols.push_back(int(v - 1));
        }
    }
    if (nodes < 0) return set_error(B40C_ERR_INVALID_VALUE, "read_dimacs: %s: no problem line", path);
    if (arcs != declared)
        return set_error(B40C_ERR_INVALID_VALUE, "read_dimacs: %s: only %lld of %lld arcs read", path, arcs, declared);
    return coo_to_csr(nodes, rows, cols, out);
}
