"""Partitions of the reference's own hot-path tests, restated as data.

Each entry cites the fixture it mirrors.  Shapes are (x, y, z) = (A, B, C) with
(shape, chunkshape, blockshape) per operand.
"""

# tests/test_linalg_gemm.c:180-271 (iarray_arange inputs, iarray_linalg_matmul)
GEMM = [
    ("f_schunk_schunk", "f4", ((100, 170), (27, 30), (12, 7)), ((170, 21), (20, 11), (10, 5)),
     ((100, 21), (40, 3), (20, 3))),
    ("d_schunk_schunk", "f8", ((300, 670), (28, 300), (11, 31)), ((670, 210), (20, 45), (7, 12)),
     ((300, 210), (43, 11), (13, 5))),
    ("f_schunk_schunk2", "f4", ((100, 200), (10, 30), (10, 10)), ((200, 150), (25, 30), (15, 12)),
     ((100, 150), (20, 30), (11, 6))),
    ("d_schunk_schunk2", "f8", ((100, 200), (10, 30), (7, 7)), ((200, 150), (25, 30), (5, 11)),
     ((100, 150), (20, 30), (17, 7))),
]

# tests/test_linalg_gemm_transpose.c:193-215 (both operands transposed views)
GEMM_T = [
    ("f_schunk_schunk", "f4", ((170, 100), (30, 27), (7, 12)), ((21, 170), (11, 20), (5, 10)),
     ((100, 21), (40, 3), (20, 3))),
]

# tests/test_linalg_gemv.c:176-246 (iarray_linspace(0, 10) inputs)
GEMV = [
    ("d_schunk", "f4", ((100, 200), (30, 30), (10, 15)), ((200,), (125,), (45,)), ((100,), (80,), (37,))),
    ("f_schunk_schunk", "f8", ((650, 900), (200, 140), (20, 14)), ((900,), (421,), (55,)),
     ((650,), (155,), (47,))),
    ("d_schunk_schunk", "f8", ((60, 300), (14, 200), (5, 14)), ((300,), (41,), (17,)), ((60,), (18,), (18,))),
]

# tests/test_linalg_gemv_transpose.c:184-207 (A transposed view)
GEMV_T = [
    ("d_schunk", "f4", ((200, 100), (30, 30), (15, 10)), ((200,), (125,), (45,)), ((100,), (80,), (37,))),
]

# tests/test_opt_gemv.c:179-225 (iarray_opt_gemv, matched partitions)
OPT_GEMV = [
    ("f_schunk", "f4", ((6000, 4000), (2000, 1000), (200, 200)), ((4000,), (1000,), (200,)),
     ((6000,), (2000,), (200,))),
    ("d_schunk", "f8", ((8000, 2000), (400, 300), (200, 150)), ((2000,), (300,), (150,)),
     ((8000,), (400,), (200,))),
]

# Reference tolerances: elementwise relative 1e-14 (f64) / 1e-5 (f32),
# tests/test_linalg_gemm.c:128-147.
TOL = {"f8": 1e-14, "f4": 1e-5}
