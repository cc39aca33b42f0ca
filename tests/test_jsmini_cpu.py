"""The JS-subset translator that produced the golden vectors keeps the JS
semantics the solver depends on, and rejects what it does not understand."""
import math

import numpy as np
import pytest

from golden import jsmini


def run(src, name="f", *args):
    ns = jsmini.load([("t.js", src)])
    return ns[name](*args)


def test_float32_store_rounds_and_load_widens():
    src = """
    function f(x) { const a = new Float32Array(2); a[0] = x; return a[0] + 0.0; }
    """
    x = 0.1
    assert run(src, "f", x) == float(np.float32(x))


def test_int32_and_truncation():
    src = "function f(p) { return (p * 255) | 0; } function g(x) { return x | 0; }"
    ns = jsmini.load([("t.js", src)])
    assert ns["f"](0.999) == 254
    assert ns["g"](-1.5) == -1
    assert ns["g"](float("nan")) == 0 and ns["g"](float("inf")) == 0
    assert ns["g"](2.0 ** 33 + 5) == 5 and ns["g"](2.0 ** 31) == -2 ** 31


def test_no_reassociation_or_comparison_chaining():
    src = "function f(a, b, c) { return a + b + c; } function g(a, b, c) { return a < b < c; }"
    ns = jsmini.load([("t.js", src)])
    assert ns["f"](1e16, -1e16, 1.0) == (1e16 + -1e16) + 1.0
    # JS: (3 < 2) < 1  ->  false < 1  ->  true ; Python chaining would give False
    assert ns["g"](3, 2, 1) is True


def test_math_semantics():
    src = """
    function f(a, b) { return Math.min(a, b); }
    function g(x) { return Math.sqrt(x); }
    """
    ns = jsmini.load([("t.js", src)])
    assert math.isnan(ns["f"](float("nan"), 1.0)) and math.isnan(ns["f"](1.0, float("nan")))
    assert math.isnan(ns["g"](-1.0))


def test_for_continue_runs_update_and_postfix_index():
    src = """
    function f(n) {
      const out = new Uint8Array(2 * n); let o = 0;
      for (let i = 0; i < n; i++) { out[o++] = i; out[o++] = 2 * i; }
      let s = 0;
      for (let j = n; j > 0; j--) { if (j % 2 === 0) continue; s += j; }
      return [out, s];
    }
    """
    out, s = run(src, "f", 4)
    assert list(out) == [0, 0, 1, 2, 2, 4, 3, 6] and s == 4


def test_class_destructuring_and_nullish():
    src = """
    class A {
      constructor(n, opts = {}) { this.n = n; this.v = opts.v ?? 7; }
      get2() { const { n, v } = this; return n * v; }
    }
    """
    ns = jsmini.load([("t.js", src)])
    assert ns["A"](3).get2() == 21
    assert ns["A"](3, jsmini._JSObject(v=2)).get2() == 6


@pytest.mark.parametrize("src", [
    "const f = (x) => x;",
    "function f(a) { for (const k of a) {} }",
    "function f(x) { { const y = 1; { const y = 2; } } }",
    "function f(a) { return a?.b; }",
])
def test_rejects_outside_the_subset(src):
    with pytest.raises(jsmini.JSSyntaxError):
        jsmini.translate(src)
