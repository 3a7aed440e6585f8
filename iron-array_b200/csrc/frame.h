// Blosc2 contiguous frame (de)serialisation for containers of this library.
#pragma once
#include <stdint.h>

#include <string>
#include <utility>
#include <vector>

namespace iab {

struct FrameInfo {
    int ndim = 0;
    int64_t shape[8] = {0}, chunk[8] = {0}, block[8] = {0};
    int dtype = 0;         // iarray_data_type_t
    int typesize = 0;
    int64_t nbytes = 0;    // uncompressed bytes of all chunks
    int32_t blocksize = 0; // bytes
    int32_t chunksize = 0; // bytes of one (padded) chunk
    int codec = 1, clevel = 5, nthreads = 1;
    bool shuffle = true;
    // sparse (directory) frame: the frame holds no chunk bytes, its offsets are chunk file
    // numbers (c-blosc2's sframe: <urlpath>/chunks.b2frame + <urlpath>/%08X.chunk)
    bool sparse = false;
};

bool write_frame(const FrameInfo &fi, const std::vector<const uint8_t *> &chunks, const std::vector<int32_t> &lens,
                 std::vector<uint8_t> *out);
// The frame pieces around the chunk bytes: header (depends on the total frame size) and
// tail (offsets chunk + trailer).  A frame is header | chunks back to back | tail.
// With fi.sparse, the header of a sparse frame's index file and a tail whose offsets are
// the chunk file numbers.
std::vector<uint8_t> frame_header(const FrameInfo &fi, int64_t data_cbytes, int64_t nchunks);
std::vector<uint8_t> frame_tail(const std::vector<int32_t> &lens, bool sparse = false);
// Parses a frame; `chunks` receives (byte offset in the frame, cbytes) in logical order, or,
// for a sparse frame's index file (fi->sparse set), (chunk file number, 0).
bool read_frame(const uint8_t *buf, size_t n, FrameInfo *fi, std::vector<std::pair<int64_t, int32_t>> *chunks,
                std::string *why);
std::vector<uint8_t> caterva_meta(int ndim, const int64_t *shape, const int64_t *chunk, const int64_t *block);
std::vector<uint8_t> iarray_meta(int dtype);

}  // namespace iab
