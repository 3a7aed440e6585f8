"""Element-wise expressions (iarray_expr_* / iarray_eval) on the GPU, through the C ABI.

The fixtures restate the reference's own tests: tests/test_expression_eval_double.c
(x[i] = i / n, each expression compared with the C math library within atol 5e-15 +
rtol 5e-14) and tests/test_expression_eval_float.c (atol 5e-3, rtol 1e-5).  The library keeps
containers at one or two dimensions, so the reference's 3-, 4- and 6-dimensional fixtures are
evaluated here on two-dimensional shapes with the same expressions.  The product epilogue
(iarray_b200_expr_bind_matmul) is checked against numpy.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (expression, numpy function of x, shape, chunkshape, blockshape); test_expression_eval_double.c
DOUBLE = [
    ("2.3", lambda x: np.full_like(x, 2.3), (100, 40), (50, 20), (15, 20)),                    # :150-162
    ("(x - 2.3) * (x - 1.35) * (x + 4.2)", lambda x: (x - 2.3) * (x - 1.35) * (x + 4.2),
     (100, 40), (50, 20), (15, 20)),                                                            # :165-177
    ("(abs(-x) - 1.35) * ceil(x) * floor(x - 8.5)",
     lambda x: (np.abs(-x) - 1.35) * np.ceil(x) * np.floor(x - 8.5), (100, 100), (25, 25), (10, 10)),  # :211-228
    ("(x - 1.35) + sin(.45)", lambda x: (x - 1.35) + np.sin(.45), (100, 100), (25, 25), (10, 10)),    # :230-248
    ("(x - 1.35) + sin(.45)", lambda x: (x - 1.35) + np.sin(.45), (100,), (25,), (10,)),              # :250-263
    ("sinh(x) + (cosh(x) - 1.35) - tanh(x + .2)",
     lambda x: np.sinh(x) + (np.cosh(x) - 1.35) - np.tanh(x + .2), (100, 100), (25, 25), (10, 10)),   # :265-282
    ("asin(x) + (acos(x) - 1.35) - atan(x + .2)",
     lambda x: np.arcsin(x) + (np.arccos(x) - 1.35) - np.arctan(x + .2), (120, 114), (24, 35), (12, 15)),  # :284-301
    ("arcsin(x) + (arccos(x) - 1.35) - arctan(x + .2)",
     lambda x: np.arcsin(x) + (np.arccos(x) - 1.35) - np.arctan(x + .2), (400, 285), (100, 209), (50, 38)),  # :303-315
    ("sin(x) * sin(x) + cos(x) * cos(x)", lambda x: np.sin(x) ** 2 + np.cos(x) ** 2,
     (400, 285), (240, 209), (50, 14)),                                                         # :317-334
    ("atan2(x, 2)", lambda x: np.arctan2(x, 2), (20000,), (2000,), (200,)),                   # :336-353
    ("pow(x, 2)", lambda x: np.power(x, 2), (20000,), (2000,), (200,)),                        # :355-372
    ("power(x, 3.141592)", lambda x: np.power(x, 3.141592), (20000,), (2000,), (200,)),        # :374-391
    ("min(x, 234.345)", lambda x: np.minimum(x, 234.345), (20000,), (2000,), (200,)),         # :393-410
    ("max(x, 4.345)", lambda x: np.maximum(x, 4.345), (20000,), (2000,), (200,)),             # :412-429
]

# test_expression_eval_float.c
FLOAT = [
    ("(abs(-x) - 1.35) * ceil(x) * floor(x - 8.5)",
     lambda x: (np.abs(-x) - 1.35) * np.ceil(x) * np.floor(x - 8.5), (100, 100), (25, 25), (10, 10)),
    ("(x - 1.35) + sin(.45)", lambda x: (x - 1.35) + np.sin(.45), (100, 100), (25, 25), (10, 10)),
    ("sinh(x) + (cosh(x) - 1.35) - tanh(x + .2)",
     lambda x: np.sinh(x) + (np.cosh(x) - 1.35) - np.tanh(x + .2), (100, 100), (25, 25), (10, 10)),
    ("asin(x) + (acos(x) - 1.35) - atan(x + .2)",
     lambda x: np.arcsin(x) + (np.arccos(x) - 1.35) - np.arctan(x + .2), (100, 100), (25, 25), (10, 10)),
    ("exp(x) + (log(x) - 1.35) - log10(x + .2)",
     lambda x: np.exp(x) + (np.log(x) - 1.35) - np.log10(x + .2), (100, 100), (25, 25), (10, 10)),
    ("2.71828**x / x * log(x)", lambda x: 2.71828 ** x / x * np.log(x), (100, 100), (25, 25), (10, 10)),
]


def _x(shape, dtype):
    n = int(np.prod(shape))
    return (np.arange(n, dtype=np.float64) * (1.0 / n)).astype(dtype).reshape(shape)


def _close(got, want, atol, rtol):
    both_inf = np.isinf(got) & np.isinf(want) & (np.sign(got) == np.sign(want))
    both_nan = np.isnan(got) & np.isnan(want)
    ok = both_inf | both_nan | (np.abs(got - want) <= atol + rtol * np.abs(want))
    assert ok.all(), (np.argwhere(~ok)[:5], got[~ok][:5], want[~ok][:5])


def _eval(ia, ctx, text, shape, cs, bs, dtype, bind_x=True):
    x = _x(shape, dtype)
    c = ia.Container.from_numpy(ctx, x, cs, bs)
    e = ia.Expression(ctx, dtype)
    if bind_x:
        e.bind("x", c)
    e.bind_out(shape, dtype, cs, bs)
    e.compile(text)
    out = e.eval().to_numpy()
    e.free()
    return x, out


@pytest.mark.parametrize("fx", DOUBLE, ids=lambda f: f[0])
def test_expression_double_reference_fixtures(ctx, ia, fx):
    text, fn, shape, cs, bs = fx
    x, out = _eval(ia, ctx, text, shape, cs, bs, np.float64, bind_x=text != "2.3")
    with np.errstate(all="ignore"):
        _close(out, fn(x), 5e-15, 5e-14)


@pytest.mark.parametrize("fx", FLOAT, ids=lambda f: f[0])
def test_expression_float_reference_fixtures(ctx, ia, fx):
    text, fn, shape, cs, bs = fx
    x, out = _eval(ia, ctx, text, shape, cs, bs, np.float32)
    with np.errstate(all="ignore"):
        want = fn(x.astype(np.float64)).astype(np.float32)
    _close(out.astype(np.float64), want.astype(np.float64), 5e-3, 1e-5)


def test_expression_several_operands_scalars_and_views(ctx, ia):
    rng = np.random.default_rng(51)
    a, b = rng.uniform(-1, 1, (90, 70)), rng.uniform(0.5, 2, (70, 90))
    ca = ia.Container.from_numpy(ctx, a, (40, 30), (20, 15))
    cb = ia.Container.from_numpy(ctx, b, (30, 40), (15, 20)).transpose()      # a 90 x 70 view
    e = ia.Expression(ctx)
    e.bind("a", ca)
    e.bind("b", cb)
    e.bind_scalar("s", 0.5)
    e.bind_out((90, 70), np.float64, (32, 32), (16, 16))
    e.compile("s * a ** 2 - sqrt(b) / (1 + exp(-a)) + max(a, -b)")
    got = e.eval().to_numpy()
    bt = b.T
    want = 0.5 * a ** 2 - np.sqrt(bt) / (1 + np.exp(-a)) + np.maximum(a, -bt)
    _close(got, want, 1e-14, 1e-14)
    # rebinding a scalar takes effect at the next compile
    e.bind_scalar("s", 2.0)
    e.compile("s * a")
    _close(e.eval().to_numpy(), 2.0 * a, 0, 0)
    e.free()


@pytest.mark.parametrize("form", ["native", "split"])
def test_expression_as_matmul_epilogue(ia, form):
    rng = np.random.default_rng(52)
    A, B, bias = rng.uniform(-1, 1, (300, 257)), rng.uniform(-1, 1, (257, 200)), rng.uniform(-1, 1, (300, 200))
    ctx = ia.Context()
    if form == "split":
        ctx.set_form(ia.FORM_SPLIT)
    ca = ia.Container.from_numpy(ctx, A, (128, 128), (32, 32))
    cb = ia.Container.from_numpy(ctx, B, (128, 128), (32, 32))
    cbias = ia.Container.from_numpy(ctx, bias, (100, 100), (50, 50))
    e = ia.Expression(ctx)
    e.bind_matmul("ab", ca, cb)
    e.bind("bias", cbias)
    e.bind_scalar("alpha", 1.5)
    e.bind_out((300, 200), np.float64, (128, 100), (32, 50))
    e.compile("max(alpha * ab + bias, 0)")
    got = e.eval().to_numpy()
    want = np.maximum(1.5 * (A @ B) + bias, 0)
    _close(got, want, 1e-13, 1e-13)
    e.free()
    ctx.close()


def test_expression_errors(ctx, ia):
    x = ia.Container.from_numpy(ctx, _x((50, 40), np.float64), (25, 20), (5, 20))
    e = ia.Expression(ctx)
    e.bind("x", x)
    for bad in ("x +", "y * 2", "sin(x, 2)", "foo(x)", "(x * 2", "x $ 2"):
        with pytest.raises(ia.IArrayError) as err:
            e.compile(bad)
        assert err.value.name == "INVALID_ARGUMENT", bad
    e.bind_out((40, 50), np.float64, (20, 25), (5, 25))       # shape differs from x's
    e.compile("x * 2")
    with pytest.raises(ia.IArrayError) as err:
        e.eval()
    assert err.value.name == "INVALID_SHAPE"
    with pytest.raises(ia.IArrayError) as err:
        ia.check(ia.lib().iarray_expr_compile_udf(e.ptr, 0, b"", b"f"), "udf")
    assert err.value.name == "NOT_SUPPORTED"
    e.free()
