// maxflow_b200 — drop-in CLI for the reference program
// (Region_Aware_PR_with_Pruning_BoundaryCore.cu main, RA:2561-2933):
//
//   maxflow_b200 <input_dir> <output_dir> [static|dynamic] [--batch] [--R N]
//                [--csr-cache FILE]
//
// Reads <input_dir>/graph.txt and test.txt (1-based ids), writes
// <output_dir>/res_mt.txt (static) or res_dynamic.txt (dynamic), one
// "flow time_ms" line per query in input order; invalid queries or s == t
// give "0 0" (RA:2659-2663).  Diagnostics go to stderr.
//   static   one plain whole-GPU solve per query (time_ms = that solve's
//            wall time, prune included, as in RA:2808).
//   --batch  all queries in one batched launch; time_ms = launch wall time
//            divided evenly over the queries.
//   dynamic  queries in windows of 10 (RA:2852), each window a resident
//            session whose residual state stays on the GPU.
//   --csr-cache FILE  load the partitioned graph from FILE (binary CSR
//            cache) when it holds one with the same R; otherwise build it
//            from graph.txt and write FILE.
//
//   maxflow_b200 --scc-contract <input_graph.txt> <output_graph_scc.txt>
//
// Drop-in for the reference's SCC tool (SCC_CONTRACT/scc_contract.cpp):
// writes the contracted graph ("n' m'" then "cu cv cap" lines, increasing
// (cu, cv)) and <output>.map ("vertex component" lines), 1-based, with the
// components computed on the GPU (mf_graph_scc) and numbered in the order
// of their smallest vertex id.
//
//   maxflow_b200 --scc-convert-test <test.txt> <graph_scc.txt.map> <out_test_scc.txt>
//   maxflow_b200 --scc-split-queries <test.txt> <graph_scc.txt.map> <test_inter.txt> <test_intra.txt>
//
// The reference's two query tools over a .map file (SCC_CONTRACT/
// convert_test_to_scc.cpp, split_queries_by_scc.cpp): each query's ends
// mapped to their components ("0 0" for an end outside the map), or the
// queries split into those whose ends lie in different components (written
// as component ids, or as given when an end is not mapped) and those inside
// one component (written as given), with <test_inter.txt>.index listing
// "query class line" per query.  Host-only text work (no device call).
#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/maxflow_b200.h"

static double now_ms() {
    return std::chrono::duration<double, std::milli>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

static int scc_main(const char *in, const char *out) {
    mf_graph *g = nullptr;
    if (mf_graph_load_file(in, 1, &g) != MF_OK) {
        fprintf(stderr, "Cannot load %s: %s\n", in, mf_last_error_string());
        return 1;
    }
    int n = 0;
    mf_graph_info(g, &n, nullptr, nullptr);
    std::vector<int32_t> comp((size_t)std::max(n, 1));
    int32_t nc = 0;
    long long mc = 0;
    if (mf_graph_scc(g, comp.data(), &nc, &mc) != MF_OK) {
        fprintf(stderr, "SCC failed: %s\n", mf_last_error_string());
        mf_graph_destroy(g);
        return 1;
    }
    std::vector<int32_t> cu((size_t)std::max(mc, 1LL)), cv(cu.size());
    std::vector<int64_t> cc(cu.size());
    int rc = mf_graph_scc_contracted(g, cu.data(), cv.data(), cc.data(), (long long)cu.size());
    mf_graph_destroy(g);
    if (rc != MF_OK) {
        fprintf(stderr, "SCC contraction failed: %s\n", mf_last_error_string());
        return 1;
    }
    fprintf(stderr, "[SCC] n=%d, components C=%d, contracted arcs m'=%lld\n", n, nc, mc);
    FILE *f = fopen(out, "w");
    if (!f) {
        fprintf(stderr, "Cannot open %s for write\n", out);
        return 1;
    }
    fprintf(f, "%d %lld\n", nc, mc);
    for (long long i = 0; i < mc; ++i)
        fprintf(f, "%d %d %lld\n", cu[i] + 1, cv[i] + 1, (long long)cc[i]);
    fclose(f);
    std::string mp = std::string(out) + ".map";
    if (FILE *m = fopen(mp.c_str(), "w")) {
        for (int i = 0; i < n; ++i) fprintf(m, "%d %d\n", i + 1, comp[i] + 1);
        fclose(m);
    }
    return 0;
}

// "vertex component" pairs (1-based) until the first line that does not
// scan; a vertex listed twice keeps its last component.  comp[v] = -1 for a
// vertex in [1, max] the map does not list.
static bool read_scc_map(const char *path, std::vector<int> &comp, int &max_v) {
    FILE *f = fopen(path, "r");
    if (!f) return false;
    std::vector<std::pair<int, int>> pairs;
    int a, b;
    max_v = 0;
    while (fscanf(f, "%d %d", &a, &b) == 2) {
        if (a < 0) continue;  // not a vertex id
        pairs.push_back({a, b});
        max_v = std::max(max_v, a);
    }
    fclose(f);
    comp.assign((size_t)max_v + 1, -1);
    for (auto &p : pairs) comp[(size_t)p.first] = p.second;
    return true;
}

static int scc_convert_main(const char *test, const char *map, const char *out) {
    std::vector<int> comp;
    int max_v = 0;
    if (!read_scc_map(map, comp, max_v)) {
        fprintf(stderr, "Cannot open %s\n", map);
        return 1;
    }
    FILE *tf = fopen(test, "r");
    if (!tf) {
        fprintf(stderr, "Cannot open %s\n", test);
        return 1;
    }
    FILE *of = fopen(out, "w");
    if (!of) {
        fclose(tf);
        fprintf(stderr, "Cannot open %s for write\n", out);
        return 1;
    }
    int u, v;
    while (fscanf(tf, "%d %d", &u, &v) == 2) {
        const bool in = u > 0 && u <= max_v && v > 0 && v <= max_v;
        const int cu = in ? comp[(size_t)u] : 0, cv = in ? comp[(size_t)v] : 0;
        if (cu > 0 && cv > 0) fprintf(of, "%d %d\n", cu, cv);
        else fprintf(of, "0 0\n");
    }
    fclose(tf);
    fclose(of);
    return 0;
}

static int scc_split_main(const char *test, const char *map, const char *inter, const char *intra) {
    std::vector<int> comp;
    int max_v = 0;
    if (!read_scc_map(map, comp, max_v)) {
        fprintf(stderr, "Cannot open %s\n", map);
        return 1;
    }
    FILE *tf = fopen(test, "r");
    if (!tf) {
        fprintf(stderr, "Cannot open %s\n", test);
        return 1;
    }
    FILE *fi = fopen(inter, "w"), *fa = fopen(intra, "w");
    if (!fi || !fa) {
        if (fi) fclose(fi);
        if (fa) fclose(fa);
        fclose(tf);
        fprintf(stderr, "Cannot open the output query files\n");
        return 1;
    }
    FILE *ix = fopen((std::string(inter) + ".index").c_str(), "w");
    int u, v, q = 0, ni = 0, na = 0;
    while (fscanf(tf, "%d %d", &u, &v) == 2) {
        ++q;
        const bool in = u > 0 && u <= max_v && v > 0 && v <= max_v;
        const int cu = in ? comp[(size_t)u] : 0, cv = in ? comp[(size_t)v] : 0;
        if (cu > 0 && cv > 0 && cu == cv) {
            fprintf(fa, "%d %d\n", u, v);  // one component: the original graph's ids
            if (ix) fprintf(ix, "%d intra %d\n", q, ++na);
            continue;
        }
        if (cu > 0 && cv > 0) fprintf(fi, "%d %d\n", cu, cv);  // across components: their ids
        else fprintf(fi, "%d %d\n", u, v);                     // an end the map does not list
        if (ix) fprintf(ix, "%d inter %d\n", q, ++ni);
    }
    fclose(tf);
    fclose(fi);
    fclose(fa);
    if (ix) fclose(ix);
    fprintf(stderr, "[Split] total queries=%d, inter=%d, intra=%d\n", q, ni, na);
    return 0;
}

int main(int argc, char **argv) {
    if (argc == 4 && !strcmp(argv[1], "--scc-contract")) return scc_main(argv[2], argv[3]);
    if (argc == 5 && !strcmp(argv[1], "--scc-convert-test")) return scc_convert_main(argv[2], argv[3], argv[4]);
    if (argc == 6 && !strcmp(argv[1], "--scc-split-queries"))
        return scc_split_main(argv[2], argv[3], argv[4], argv[5]);
    if (argc < 3) {
        fprintf(stderr, "Usage: %s <input_dir> <output_dir> [mode] [--batch] [--R N] [--csr-cache FILE]\n",
                argv[0]);
        fprintf(stderr, "  mode = static (default) | dynamic\n");
        fprintf(stderr, "   or: %s --scc-contract <input_graph.txt> <output_graph_scc.txt>\n", argv[0]);
        fprintf(stderr, "   or: %s --scc-convert-test <test.txt> <graph_scc.txt.map> <out_test_scc.txt>\n", argv[0]);
        fprintf(stderr, "   or: %s --scc-split-queries <test.txt> <graph_scc.txt.map> <test_inter.txt> <test_intra.txt>\n",
                argv[0]);
        return 1;
    }
    std::string in = argv[1], outd = argv[2], mode = "static";
    bool batch = false;
    int R = 128;  // RA:2583
    std::string cache;
    for (int i = 3; i < argc; ++i) {
        if (!strcmp(argv[i], "--batch")) batch = true;
        else if (!strcmp(argv[i], "--R") && i + 1 < argc) R = atoi(argv[++i]);
        else if (!strcmp(argv[i], "--csr-cache") && i + 1 < argc) cache = argv[++i];
        else mode = argv[i];
    }
    if (mode != "static" && mode != "dynamic") {
        fprintf(stderr, "Unknown mode: %s (use static or dynamic)\n", mode.c_str());
        return 1;
    }
    mkdir(outd.c_str(), 0755);
    mf_graph *g = nullptr;
    double t0 = now_ms();
    int rc = MF_ERR_IO;
    bool from_cache = false;
    if (!cache.empty() && mf_graph_load_binary(cache.c_str(), &g) == MF_OK) {
        int cn = 0, cR = 0;
        long long ca = 0;
        mf_graph_info(g, &cn, &ca, &cR);
        // the R a build from graph.txt would use (0 -> 128, clamped to [1, min(n, 1024)])
        int want = R <= 0 ? 128 : R;
        want = std::min(std::min(want, cn), 1024);
        if (cR == want) {
            from_cache = true;
            rc = MF_OK;
        } else {
            mf_graph_destroy(g);
            g = nullptr;
        }
    }
    if (!from_cache) {
        rc = mf_graph_load_file((in + "/graph.txt").c_str(), R, &g);
        if (rc != MF_OK) {
            fprintf(stderr, "Cannot load %s/graph.txt: %s\n", in.c_str(), mf_last_error_string());
            return 1;
        }
        if (!cache.empty() && mf_graph_save(g, cache.c_str()) != MF_OK)
            fprintf(stderr, "Cannot write the CSR cache %s: %s\n", cache.c_str(), mf_last_error_string());
    }
    int n = 0, Rg = 0;
    long long arcs = 0;
    mf_graph_info(g, &n, &arcs, &Rg);
    FILE *tf = fopen((in + "/test.txt").c_str(), "r");
    if (!tf) {
        fprintf(stderr, "Cannot open %s/test.txt\n", in.c_str());
        mf_graph_destroy(g);
        return 1;
    }
    std::vector<int32_t> qs, qt;
    int a, b;
    while (fscanf(tf, "%d %d", &a, &b) == 2) {
        int s = a - 1, t = b - 1;
        if (s >= 0 && s < n && t >= 0 && t < n) {
            qs.push_back(s);
            qt.push_back(t);
        } else {
            qs.push_back(-1);
            qt.push_back(-1);
        }
    }
    fclose(tf);
    fprintf(stderr, "Graph (reordered by Region): n=%d, m=%lld, Regions=%d, Queries=%zu (load %.0f ms)\n",
            n, arcs, Rg, qs.size(), now_ms() - t0);
    const size_t Q = qs.size();
    std::vector<long long> flows(Q, 0), times(Q, 0);
    mf_opts o;
    mf_opts_default(&o);
    int status = 0;
    if (mode == "static") {
        if (batch && Q > 0) {
            double b0 = now_ms();
            std::vector<int64_t> f(Q);
            rc = mf_solve_batch(g, (int)Q, qs.data(), qt.data(), &o, f.data(), nullptr);
            double el = now_ms() - b0;
            if (rc != MF_OK) {
                fprintf(stderr, "batch solve failed: %s\n", mf_last_error_string());
                status = 1;
            }
            for (size_t i = 0; i < Q; ++i) {
                bool valid = qs[i] >= 0 && qs[i] != qt[i];
                flows[i] = valid ? f[i] : 0;
                times[i] = valid ? (long long)(el / Q) : 0;
            }
            fprintf(stderr, "[Batch] %zu queries in %.3f ms\n", Q, el);
        } else {
            for (size_t i = 0; i < Q; ++i) {
                if (qs[i] < 0 || qs[i] == qt[i]) {
                    fprintf(stderr, "[Static] Query %zu: Invalid.\n", i + 1);
                    continue;
                }
                mf_stats st;
                int64_t f = 0;
                double q0 = now_ms();
                rc = mf_solve(g, qs[i], qt[i], &o, &f, &st);
                double el = now_ms() - q0;
                if (rc != MF_OK) {
                    fprintf(stderr, "query %zu failed: %s\n", i + 1, mf_last_error_string());
                    status = 1;
                }
                flows[i] = f;
                times[i] = (long long)el;
                fprintf(stderr,
                        "[Static] Query %zu: s=%d, t=%d kept_n=%d, kept_m=%lld, rounds=%lld, "
                        "relabels=%lld, Flow=%lld, Time=%lld ms (device %.3f ms)\n",
                        i + 1, qs[i] + 1, qt[i] + 1, st.mask_vertices, st.mask_arcs, st.rounds,
                        st.global_relabels, (long long)f, times[i], st.time_ms);
            }
        }
        std::string res = outd + "/res_mt.txt";
        FILE *out = fopen(res.c_str(), "w");
        if (!out) {
            fprintf(stderr, "Cannot open output file %s\n", res.c_str());
            mf_graph_destroy(g);
            return 1;
        }
        long long total = 0;
        for (size_t i = 0; i < Q; ++i) {
            fprintf(out, "%lld %lld\n", flows[i], times[i]);
            total += times[i];
        }
        fclose(out);
        fprintf(stderr, "Total time: %lld ms\n", total);
    } else {
        std::string res = outd + "/res_dynamic.txt";
        FILE *out = fopen(res.c_str(), "w");
        if (!out) {
            fprintf(stderr, "Cannot open dynamic output file %s\n", res.c_str());
            mf_graph_destroy(g);
            return 1;
        }
        const size_t WINDOW = 10;  // RA:2852
        long long total = 0;
        for (size_t q0 = 0; q0 < Q; q0 += WINDOW) {
            size_t q1 = std::min(Q, q0 + WINDOW);
            std::vector<int32_t> ws, wt;
            std::vector<size_t> idx;
            for (size_t i = q0; i < q1; ++i)
                if (qs[i] >= 0 && qs[i] != qt[i]) {
                    ws.push_back(qs[i]);
                    wt.push_back(qt[i]);
                    idx.push_back(i);
                }
            if (!ws.empty()) {
                mf_session *ss = nullptr;
                double w0 = now_ms();
                rc = mf_session_create(g, (int)ws.size(), ws.data(), wt.data(), &o, &ss);
                std::vector<int64_t> f(ws.size(), 0);
                if (rc == MF_OK) rc = mf_session_solve(ss, f.data(), nullptr);
                double el = now_ms() - w0;
                if (rc != MF_OK) {
                    fprintf(stderr, "window [%zu,%zu) failed: %s\n", q0, q1, mf_last_error_string());
                    status = 1;
                }
                for (size_t k = 0; k < idx.size(); ++k) {
                    flows[idx[k]] = f[k];
                    times[idx[k]] = (long long)(el / idx.size());
                }
                mf_session_destroy(ss);
            }
            for (size_t i = q0; i < q1; ++i) {
                fprintf(out, "%lld %lld\n", flows[i], times[i]);
                total += times[i];
            }
        }
        fclose(out);
        fprintf(stderr, "Total time: %lld ms\n", total);
    }
    mf_graph_destroy(g);
    return status;
}
