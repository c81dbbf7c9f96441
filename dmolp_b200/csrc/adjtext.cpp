// Parallel loader for the reference's adjacency text (src/phase1/init.cpp:8-100): first line = V, then one
// line per vertex with its neighbour ids.  Produces the CSR the reference builds from it
// (src/phase1/partition.cpp:227-262: each row sorted and de-duplicated, self-loops kept) plus the raw
// per-line token count that phase 1 uses as the degree.
//
// Tokenisation is the reference's fast_atoi (init.cpp:15-23): read a run of digits (possibly empty, giving
// 0), then skip non-digits; a line is parsed until its end or a NUL byte.  A final line without '\n' is
// dropped, as the reference's block reader drops it (init.cpp:214-243).  The vertex count is the number of
// newline-terminated lines after the header (the reference uses adj.size()); a neighbour id outside
// [0, V) is rejected (the reference would index its bitsets out of range).  Unlike the reference, lines
// longer than its 16 MiB read block are read correctly.
#include <omp.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "adjtext.hpp"

namespace {
thread_local std::string g_err;
}

struct dmolp_host_graph {
    std::vector<int64_t> off;
    std::vector<int32_t> col;
    std::vector<int32_t> raw;
};

extern "C" {

const char *dmolp_adjtext_error(void) { return g_err.c_str(); }

int dmolp_adjtext_load(const char *path, dmolp_host_graph **out) {
    FILE *f = fopen(path, "rb");
    if (!f) {
        g_err = std::string("cannot open ") + path;
        return 1;
    }
    fseek(f, 0, SEEK_END);
    const long long size = ftell(f);
    fseek(f, 0, SEEK_SET);
    std::vector<char> data((size_t)size + 1);
    if (size > 0 && fread(data.data(), 1, (size_t)size, f) != (size_t)size) {
        fclose(f);
        g_err = "short read";
        return 1;
    }
    fclose(f);
    data[size] = '\0';
    const char *buf = data.data();
    const char *hdr_end = (const char *)memchr(buf, '\n', (size_t)size);
    if (!hdr_end) {
        g_err = "missing header line";
        return 1;
    }
    const size_t body0 = (size_t)(hdr_end - buf) + 1;
    // last newline: anything after it is an unterminated line and is dropped
    size_t body1 = (size_t)size;
    while (body1 > body0 && buf[body1 - 1] != '\n') --body1;

    const int T = std::max(1, omp_get_max_threads());
    std::vector<size_t> cb(T + 1);
    cb[0] = body0;
    cb[T] = body1;
    for (int t = 1; t < T; ++t) {
        size_t p = body0 + (body1 - body0) * t / T;
        if (p < cb[t - 1]) p = cb[t - 1];
        while (p < body1 && p > body0 && buf[p - 1] != '\n') ++p;
        cb[t] = p;
    }
    std::vector<int64_t> lines(T + 1, 0);
#pragma omp parallel for num_threads(T) schedule(static, 1)
    for (int t = 0; t < T; ++t) {
        int64_t n = 0;
        for (size_t i = cb[t]; i < cb[t + 1]; ++i) n += buf[i] == '\n';
        lines[t + 1] = n;
    }
    for (int t = 0; t < T; ++t) lines[t + 1] += lines[t];
    const int64_t nv = lines[T];
    if (nv > 0x7ffffffe) {
        g_err = "too many vertices for int32 ids";
        return 1;
    }
    dmolp_host_graph *g = new dmolp_host_graph();
    g->raw.assign(nv, 0);
    std::vector<int64_t> ucount(nv + 1, 0);
    std::vector<std::vector<int32_t>> chunk_cols(T);
    int bad = 0;
#pragma omp parallel for num_threads(T) schedule(static, 1) reduction(| : bad)
    for (int t = 0; t < T; ++t) {
        std::vector<int32_t> &cc = chunk_cols[t];
        std::vector<int64_t> row;
        int64_t v = lines[t];
        size_t i = cb[t];
        while (i < cb[t + 1]) {
            row.clear();
            // one line: [i, newline)
            while (buf[i] != '\n' && buf[i] != '\0') {
                int64_t x = 0;
                while ((unsigned)(buf[i] - '0') <= 9) x = x * 10 + (buf[i++] - '0');
                while (buf[i] != '\n' && buf[i] != '\0' && (unsigned)(buf[i] - '0') > 9) ++i;
                row.push_back(x);
            }
            while (buf[i] != '\n') ++i;  // a NUL ends the parse of this line (as c_str() would)
            ++i;
            g->raw[v] = (int32_t)row.size();
            std::sort(row.begin(), row.end());
            row.erase(std::unique(row.begin(), row.end()), row.end());
            for (int64_t x : row) {
                if (x < 0 || x >= nv) bad |= 1;
                cc.push_back((int32_t)x);
            }
            ucount[v + 1] = (int64_t)row.size();
            ++v;
        }
    }
    if (bad) {
        delete g;
        g_err = "a neighbour id is outside [0, V)";
        return 1;
    }
    g->off.assign(nv + 1, 0);
    for (int64_t v = 0; v < nv; ++v) g->off[v + 1] = g->off[v] + ucount[v + 1];
    g->col.resize(g->off[nv]);
#pragma omp parallel for num_threads(T) schedule(static, 1)
    for (int t = 0; t < T; ++t)
        if (!chunk_cols[t].empty())
            std::memcpy(g->col.data() + g->off[lines[t]], chunk_cols[t].data(), chunk_cols[t].size() * sizeof(int32_t));
    *out = g;
    return 0;
}

int64_t dmolp_host_graph_nv(const dmolp_host_graph *g) { return g ? (int64_t)g->raw.size() : -1; }
int64_t dmolp_host_graph_narcs(const dmolp_host_graph *g) { return g ? (int64_t)g->col.size() : -1; }
const int64_t *dmolp_host_graph_offsets(const dmolp_host_graph *g) { return g->off.data(); }
const int32_t *dmolp_host_graph_indices(const dmolp_host_graph *g) { return g->col.data(); }
const int32_t *dmolp_host_graph_raw_degree(const dmolp_host_graph *g) { return g->raw.data(); }
void dmolp_host_graph_free(dmolp_host_graph *g) { delete g; }

}  // extern "C"
