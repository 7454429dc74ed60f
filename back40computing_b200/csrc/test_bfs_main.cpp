// test_bfs: command-line driver over the drop-in C++ API, shaped like the
// reference's test/bfs/test_bfs.cu (main :903-1148, RunTests :600-756).
//
//   test_bfs <graph> <args> [--strategy=0,1,2,3] [--src=<v>|randomize] [--i=<n>]
//            [--queue-sizing=<f>] [--mark-pred] [--max-ctas=<n>] [--variant=<0|1|2>]
//            [--labels-out=<file>] [--quiet]
//   graphs: grid2d <width> | grid3d <width> | rmat <scale> <edge-factor> [<seed>]
//           | erdos <nodes> <mean-degree> [<seed>] | market <file.mtx>
//
// Strategy numbers follow test_bfs.cu:71-78 (0 expand-contract, 1
// contract-expand, 2 two-phase).  Results are checked by the package's tests
// (against the oracle), not here; --labels-out writes the int32 labels of the
// last search for them.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "b40c/graph/bfs/csr_problem.hpp"
#include "b40c/graph/bfs/enactors.hpp"
#include "b40c_bfs.h"

using namespace b40c::graph;

namespace {

struct Args {
    std::vector<std::string> pos;
    std::vector<int> strategies{0};
    std::string src = "";
    int iterations = 1;
    double queue_sizing = 1.3;  // test_bfs.cu:802
    bool mark_pred = false;
    bool quiet = false;
    int max_ctas = 0;
    int variant = B40C_VARIANT_DEFAULT;
    std::string labels_out;
};

Args parse(int argc, char **argv) {
    Args a;
    for (int i = 1; i < argc; i++) {
        std::string s = argv[i];
        auto val = [&](const char *key) -> const char * {
            size_t n = strlen(key);
            return s.compare(0, n, key) == 0 ? s.c_str() + n : nullptr;
        };
        if (const char *v = val("--strategy=")) {
            a.strategies.clear();
            for (const char *q = v; *q;) {
                a.strategies.push_back(atoi(q));
                const char *c = strchr(q, ',');
                if (!c) break;
                q = c + 1;
            }
        } else if (const char *v = val("--src=")) a.src = v;
        else if (const char *v = val("--i=")) a.iterations = atoi(v);
        else if (const char *v = val("--queue-sizing=")) a.queue_sizing = atof(v);
        else if (const char *v = val("--max-ctas=")) a.max_ctas = atoi(v);
        else if (const char *v = val("--variant=")) a.variant = atoi(v);
        else if (const char *v = val("--labels-out=")) a.labels_out = v;
        else if (s == "--mark-pred") a.mark_pred = true;
        else if (s == "--quiet") a.quiet = true;
        else a.pos.push_back(s);
    }
    return a;
}

int build_graph(const Args &a, b40c_csr_t *g, int *default_src) {
    if (a.pos.empty()) return -1;
    const std::string &t = a.pos[0];
    auto arg = [&](size_t i, long long dflt) { return i < a.pos.size() ? atoll(a.pos[i].c_str()) : dflt; };
    int rc;
    if (t == "grid2d") {
        int w = (int)arg(1, 1024);
        rc = b40c_graph_grid2d(w, 0, g);
        *default_src = (w / 2) * w + w / 2;  // grid centre
    } else if (t == "grid3d") {
        int w = (int)arg(1, 256);
        rc = b40c_graph_grid3d(w, 0, g);
        *default_src = 0;
    } else if (t == "rmat") {
        rc = b40c_graph_rmat((int)arg(1, 16), (int)arg(2, 16), 0.57, 0.19, 0.19, (uint64_t)arg(3, 1), 1, g);
        *default_src = -1;
    } else if (t == "erdos") {
        long long n = arg(1, 100000);
        rc = b40c_graph_erdos_renyi((int)n, double(arg(2, 16)) / double(n - 1), (uint64_t)arg(3, 1), g);
        *default_src = -1;
    } else if (t == "market") {
        if (a.pos.size() < 2) return -1;
        rc = b40c_graph_read_market(a.pos[1].c_str(), 1, g);
        *default_src = -1;
    } else {
        fprintf(stderr, "Unspecified graph type\n");
        return -1;
    }
    if (rc) fprintf(stderr, "graph construction failed: %s\n", b40c_last_error_string());
    return rc;
}

template <bool MP>
int run(const Args &a, b40c_csr_t &g, int default_src) {
    typedef bfs::CsrProblem<int, int, MP> Problem;
    Problem problem;
    if (problem.FromHostProblem(false, (int)g.nodes, (int)g.edges, g.column_indices, g.row_offsets, 1)) {
        fprintf(stderr, "FromHostProblem: %s\n", b40c_last_error_string());
        return 1;
    }
    bfs::EnactorExpandContract<false> expand_contract;
    bfs::EnactorContractExpand<false> contract_expand;
    bfs::EnactorTwoPhase<false> two_phase;
    bfs::EnactorHybrid<false> hybrid;
    std::vector<int> labels((size_t)g.nodes);
    std::vector<int> sources((size_t)std::max(1, a.iterations));
    if (a.src == "randomize" || (a.src.empty() && default_src < 0)) {
        b40c_graph_sample_sources(&g, (int)sources.size(), 2, sources.data());
    } else {
        int s = a.src.empty() ? default_src : atoi(a.src.c_str());
        for (auto &x : sources) x = s;
    }
    for (size_t it = 0; it < sources.size(); it++) {
        int src = sources[it];
        for (int strategy : a.strategies) {
            cudaError_t rc;
            long long total_queued = 0;
            int depth = 0;
            double duty = 0;
            auto t0 = std::chrono::steady_clock::now();
#define B40C_RUN(E)                                                                                    \
    do {                                                                                               \
        if ((rc = problem.Reset(E.GetFrontierType(), a.queue_sizing))) break;                          \
        t0 = std::chrono::steady_clock::now();                                                         \
        rc = a.variant == B40C_VARIANT_ITERATIVE ? E.EnactIterativeSearch(problem, src, a.max_ctas)   \
                                                 : E.EnactSearch(problem, src, a.max_ctas);            \
        if (!rc) E.GetStatistics(total_queued, depth, duty);                                           \
    } while (0)
            if (strategy == 0) B40C_RUN(expand_contract);
            else if (strategy == 1) B40C_RUN(contract_expand);
            else if (strategy == 2) B40C_RUN(two_phase);
            else if (strategy == 3) B40C_RUN(hybrid);
            else {
                fprintf(stderr, "strategy %d not provided\n", strategy);
                return 1;
            }
#undef B40C_RUN
            double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            if (rc) {
                fprintf(stderr, "search failed: %s (cudaError_t %d)\n", b40c_last_error_string(), (int)rc);
                return 1;
            }
            if (problem.ExtractResults(labels.data())) return 1;
            long long nv = 0, ev = 0;
            for (long long v = 0; v < g.nodes; v++)
                if (labels[(size_t)v] > -1 || (MP && labels[(size_t)v] == -2)) {
                    nv++;
                    ev += g.row_offsets[v + 1] - g.row_offsets[v];
                }
            if (!a.quiet)
                printf("[strategy %d] src %d: %.3f ms (host wall), %.3f MiEdges/s, search_depth %d, nodes visited %lld, "
                       "edges visited %lld\n",
                       strategy, src, ms, double(ev) / (ms * 1000.0), depth, nv, ev);
        }
    }
    if (!a.labels_out.empty()) {
        FILE *f = fopen(a.labels_out.c_str(), "wb");
        if (!f || fwrite(labels.data(), sizeof(int), labels.size(), f) != labels.size()) return 1;
        fclose(f);
    }
    return 0;
}

}  // namespace

int main(int argc, char **argv) {
    Args a = parse(argc, argv);
    b40c_csr_t g{};
    int default_src = 0;
    if (build_graph(a, &g, &default_src)) {
        fprintf(stderr, "usage: test_bfs <grid2d w|grid3d w|rmat scale ef [seed]|erdos n deg [seed]|market file> "
                        "[--strategy=0,1,2,3] [--src=v|randomize] [--i=n] [--queue-sizing=f] [--mark-pred] "
                        "[--max-ctas=n] [--variant=0|1|2] [--labels-out=file] [--quiet]\n");
        return 1;
    }
    int rc = a.mark_pred ? run<true>(a, g, default_src) : run<false>(a, g, default_src);
    b40c_csr_free(&g);
    return rc;
}
