// AAFL compressed column blocks: the host-side view of a block that the decoder and the fused aggregation pass read.
#pragma once

#include "qdb_common.cuh"

namespace qdb {

struct AaflView {
    const void* words = nullptr;     // the packed words (aligned to the word size)
    int64_t words_len = 0;           // words available
    const uint64_t* pos = nullptr;   // per group: index of its first word
    const uint8_t* bits = nullptr;   // per group: bits per value
    uint64_t off = 0;                // added back to every value (wrapping, in the word type)
    int64_t rows = 0;
    int64_t groups = 0;
    int word_bytes = 4;              // 4 (INT32, FLOAT) or 8 (INT64)
    void* scratch = nullptr;         // an aligned copy of the words, when the block's words start unaligned
};

// Checks a block's header counts and builds its view on `s`.  A word region that does not start on an `align`-byte
// boundary (at least the word size) is copied to an aligned scratch buffer, which the caller releases with dev_free
// after its last use on `s`.
int32_t aafl_view(const qdb_aafl_col* c, AaflView* v, cudaStream_t s, int align = 0);

}  // namespace qdb
