// Device parse of the reference's adjacency text (src/phase1/init.cpp:25-100) into the resident CSR
// (src/phase1/partition.cpp:227-262: rows sorted and de-duplicated, self-loops kept), with the raw per-line
// token count that phase 1 sorts by.  Same semantics as the host loader (adjtext.cpp); the host finds the
// header line and the last newline, everything between runs here.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace dmolp {
namespace ingest {

constexpr int kTxtThreads = 256;              // threads of the text kernels
constexpr int kChunkBytes = 16;               // bytes per thread per step (one 16-byte load)
constexpr int kTxtSteps = 4;                  // steps per tile
constexpr int64_t kTileBytes = (int64_t)kTxtThreads * kChunkBytes * kTxtSteps;  // 16 KiB of text per block
constexpr int kLineSteps = 16;                // lines per thread in the per-line kernels (block-strided)
constexpr int64_t kLineTile = (int64_t)kTxtThreads * kLineSteps;
constexpr int64_t kTokTile = 4096;            // tokens per block in the de-duplication scan

// Device text buffer size for `len` bytes: whole tiles plus one, so every 16-byte load of a tile and the
// look-ahead past a warp's window stay inside the allocation.
inline int64_t padded_bytes(int64_t len) { return (len / kTileBytes + 2) * kTileBytes; }

// Grow-only device scratch of the parse, kept by the context so that repeated loads allocate nothing
// (trimmed after a load when it holds more than kKeepScratch bytes).
enum Slot { kText, kScal, kTcnt, kToff, kTok, kTmp, kEndTok, kKeptpos, kBadrow, kLists, kLcnt, kLoff, kNumSlots };
constexpr size_t kKeepScratch = size_t(6) << 30;

struct Pool {
    void *ptr[kNumSlots] = {};
    size_t cap[kNumSlots] = {};
    // At least `bytes` bytes in `slot` (contents not kept when it grows); null with `err` set on failure.
    void *get(int slot, size_t bytes, std::string &err);
    size_t held() const;
    void release();
    void trim(size_t keep) {
        if (held() > keep) release();
    }
};

// Parse state between the sizing pass and the CSR build (device scratch borrowed from a Pool).
struct Parsed {
    int64_t nv = 0;          // newline-terminated lines after the header
    int64_t ntok = 0;        // tokens (sum of raw degrees)
    int64_t narcs = 0;       // arcs after per-row de-duplication
    int64_t maxdeg = 0, maxraw = 0;
    int64_t nb[3] = {0, 0, 0};  // vertices per degree class (1..16, 17..4096, above), degree 0 in none
    int sorted = 1;          // every row was already strictly increasing: no device sort ran
    int64_t rows_sorted = 0; // rows the device sorted
    long long launches = 0;  // kernels launched
    float count_ms = 0.f, emit_ms = 0.f;  // device time of the text count pass and of the token emit pass
    // device scratch
    uint32_t *tok = nullptr;      // [ntok] values; bit 31 marks the first token of a line
    uint32_t *tmp = nullptr;      // [ntok] merge buffer of the long-row sort (only when needed)
    int64_t *end_tok = nullptr;   // [nv] tokens before each line's newline
    int64_t *keptpos = nullptr;   // [ntok+1] arcs kept before each token (only when some row was unsorted)
    uint32_t *tcnt = nullptr;     // per-tile counters
    int64_t *toff = nullptr;      // per-tile exclusive prefixes
    int64_t *loff = nullptr;      // per-line-tile class prefixes
    uint8_t *badrow = nullptr;    // [nv] row needs sorting
    int32_t *lists = nullptr;     // rows to sort, by length class
    void *scal = nullptr;         // device counters
    Pool *pool = nullptr;
};

// Sizing pass: d_txt holds the text padded to padded_bytes(len) (padding zeroed), body = [body0, body1)
// (after the header's newline, up to and including the last newline).  NUL bytes in the body are
// overwritten in place (a NUL ends the parse of its line).  On success p holds the sizes and the scratch.
// Returns 0, or 1 with `err` set (bad id, too many vertices, CUDA failure).
int parse(cudaStream_t st, uint8_t *d_txt, int64_t len, int64_t body0, int64_t body1, Pool &pool, Parsed &p,
          std::string &err);

// A binary CSR already on the device (off[nv+1] with off[0] = 0 and off[nv] = narcs checked by the caller,
// col[narcs], raw[nv] or null): checks every row bound and id, whether every row is strictly increasing,
// and sizes the degree classes.  Synchronises the stream.  Returns 0 with `out` filled (out.bad nonzero:
// the CSR is invalid), or 1 with `err` set on a CUDA failure.
struct CsrInfo {
    int bad = 0;                // 1: offsets out of order or out of [0, narcs], 2: an id outside [0, nv), 4: raw < 0
    int sorted = 1;             // every row strictly increasing
    int64_t maxdeg = 0, maxraw = 0;
    int64_t nb[3] = {0, 0, 0};  // vertices per degree class
    int64_t *loff = nullptr;    // device per-tile class prefixes (pool scratch) for csr_classes
    long long launches = 0;
};
int check_csr(cudaStream_t st, const int64_t *off, const int32_t *col, const int32_t *raw, int64_t nv, int64_t narcs,
              Pool &pool, CsrInfo &out, std::string &err);
// The degree-class lists of a checked CSR into bucket[c][nb[c]], ascending ids.
int csr_classes(cudaStream_t st, const int64_t *off, int64_t nv, const CsrInfo &info, int32_t *const bucket[3],
                std::string &err);

// CSR build into the context's arrays: off[nv+1], col[narcs], raw[nv], and the degree-class lists
// bucket[c][nb[c]] in ascending id order.
int build(cudaStream_t st, Parsed &p, int64_t *off, int32_t *col, int32_t *raw, int32_t *const bucket[3],
          std::string &err);

void release(Parsed &p);  // returns the scratch to the pool (nothing is freed)

}  // namespace ingest
}  // namespace dmolp
