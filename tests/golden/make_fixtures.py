"""Generate the committed golden fixtures from the reference's own Blosc2 frames.

Run in a checkout where the reference is mounted (it reads
<reference>/tests/data/test_*.iarray, written by the reference toolchain via
tests/generator.py:24-76 with LZ4 clevel 5, SHUFFLE, btune off):

    python tests/golden/make_fixtures.py /path/to/reference

Outputs (committed):
  chunk_<name>_0.bin       first data chunk of three frames, byte-for-byte
  <name>.iarray            one whole frame (the smallest), byte-for-byte
  golden_digests.json      for all 10 frames: frame header / trailer bytes, and per chunk
                           the SHA-256 of the compressed chunk and of its decoded bytes,
                           its cbytes and stream-kind counts.
The decoded digests come from the oracle decoder; tests check the oracle, and through it
the GPU library, against these.
"""
import glob
import hashlib
import json
import os
import struct
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle as O  # noqa: E402

KEEP = ["test_binomial_int32_n1_p0.7", "test_poisson_int32_lam3", "test_rand_float32"]
# whole frames copied byte for byte: opened by the library itself in the GPU tests
KEEP_FRAMES = ["test_binomial_int32_n1_p0.7"]


def main(ref):
    files = sorted(glob.glob(os.path.join(ref, "tests", "data", "test_*.iarray")))
    out = {}
    for f in files:
        name = os.path.basename(f)[:-len(".iarray")]
        buf = open(f, "rb").read()
        fr = O.read_frame(buf)
        ndim, shape, chunk, block = O.parse_caterva_meta(fr["metalayers"]["caterva"])
        dtype = fr["metalayers"]["iarray"][2]
        chunks = []
        for c in fr["chunks"]:
            kinds = {"zero": 0, "run": 0, "raw": 0, "lz4": 0}
            h = O.chunk_header(c)
            for blk in O.chunk_streams(c):
                for cs, _ in blk:
                    k = "zero" if cs == 0 else "run" if cs < 0 else \
                        "raw" if cs == h["blocksize"] // h["typesize"] else "lz4"
                    kinds[k] += 1
            chunks.append(dict(cbytes=len(c), sha_chunk=hashlib.sha256(c).hexdigest(),
                               sha_decoded=hashlib.sha256(O.chunk_decompress(c)).hexdigest(),
                               kinds=kinds))
        trailer_at = fr["header_size"] + sum(len(c) for c in fr["chunks"])
        off_len = struct.unpack_from("<i", buf, trailer_at + 12)[0]
        out[name] = dict(ndim=ndim, shape=shape, chunkshape=chunk, blockshape=block,
                         iarray_dtype=dtype, typesize=fr["typesize"], blocksize=fr["blocksize"],
                         chunksize=fr["chunksize"], nbytes=fr["nbytes"], cbytes=fr["cbytes"],
                         header_hex=buf[:fr["header_size"]].hex(),
                         offsets_chunk_hex=buf[trailer_at:trailer_at + off_len].hex(),
                         trailer_hex=buf[trailer_at + off_len:].hex(),
                         chunks=chunks)
        if name in KEEP:
            with open(os.path.join(HERE, f"chunk_{name}_0.bin"), "wb") as fh:
                fh.write(fr["chunks"][0])
        if name in KEEP_FRAMES:
            with open(os.path.join(HERE, f"{name}.iarray"), "wb") as fh:
                fh.write(buf)
    with open(os.path.join(HERE, "golden_digests.json"), "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
    print(f"wrote {len(out)} frame digests, {len(KEEP)} chunks")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_fixtures.py <reference checkout (holds tests/data/*.iarray)>")
    main(sys.argv[1])
