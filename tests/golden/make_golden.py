"""Generate golden operator vectors by running sumpy's own symbolic expansion code.

This script is test infrastructure. It is run by hand in a container that has
the sumpy source tree (its path in the ``SUMPY_REFERENCE`` environment
variable, which is required) and sympy installed; the GPU test box never runs it. It writes
``tests/golden/laplace3d_operators.json``,
``tests/golden/helmholtz3d_operators.json`` and (``--which qbx``)
``tests/golden/qbx3d_pairs.json``, which the tests read
(``SUMPY_REFERENCE=<sumpy checkout> python tests/golden/make_golden.py
[--which laplace helmholtz qbx] [--laplace-orders 2 3 4 5 6 8]
[--helmholtz-orders 2 3 4] [--qbx-line-orders 3 5 8] ...``).

sumpy itself cannot be imported normally here: its package ``__init__`` pulls
in pyopencl/loopy/boxtree, none of which are installed. The expansion math
(``sumpy/expansion/{__init__,multipole,local,m2l,diff_op}.py``,
``sumpy/derivative_taker.py``, ``sumpy/kernel.py``) only needs a handful of
small utilities from ``pytools`` and ``constantdict``; everything else those
modules import is used only when generating loopy code. So this script

* installs placeholder modules for the code-generation dependencies
  (any attribute is an inert class), plus small working versions of the
  ``pytools`` helpers the math uses (``memoize_method``, ``memoize``,
  ``single_valued``, the integer-tuple generators, ``ProcessLogger``) and an
  immutable-dict ``constantdict``;
* registers a bare ``sumpy`` package object whose ``__path__`` points at the
  reference tree, so ``sumpy/__init__.py`` (which imports the OpenCL stack) is
  skipped and submodules load directly from the reference sources;
* subclasses sumpy's ``LaplaceKernel`` only to return the sympy expression
  ``1/|d|`` directly (sumpy builds it via pymbolic, ``sumpy/kernel.py:650-658``),
  leaving ``get_derivative_taker`` (``LaplaceDerivativeTaker``) and
  ``get_pde_as_diff_op`` (the Laplacian) as sumpy defines them; and sumpy's
  ``HelmholtzKernel`` (``sumpy/kernel.py:755-844``) the same way with
  ``exp(i k |d|)/|d|`` at k = 5/2, keeping ``HelmholtzDerivativeTaker``
  (``sumpy/derivative_taker.py:354-389``) and the PDE Laplacian + k^2.

For each order it then calls, on symbolic inputs, the same methods sumpy's
loopy kernels are generated from, and evaluates the results at fixed inputs
with 40-digit arithmetic:

* P2M  ``VolumeTaylorMultipoleExpansionBase.coefficients_from_source``
  (``sumpy/expansion/multipole.py:77-128``)
* P2L  ``VolumeTaylorLocalExpansionBase.coefficients_from_source``
  (``sumpy/expansion/local.py:225-282``)
* M2P  ``VolumeTaylorMultipoleExpansionBase.evaluate`` (``multipole.py:131-157``)
* L2P  ``VolumeTaylorLocalExpansionBase.evaluate`` (``local.py:284-309``)
* M2M  ``VolumeTaylorMultipoleExpansionBase.translate_from`` (``multipole.py:159-407``)
* L2L  ``VolumeTaylorLocalExpansionBase.translate_from`` (``local.py:311-493``)
* M2L  same, through ``VolumeTaylorM2LTranslation`` (the Toeplitz form,
  ``sumpy/expansion/m2l.py:363-830``), which is what the FFT form computes
  in exact arithmetic.

Kernel scaling (1/(4 pi)) is not part of these operators; sumpy applies it on
output to point values only (``MEMO``; ``sumpy/p2p.py:617``).

Usage::

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import importlib.abc
import importlib.machinery
import itertools
import json
import os
import sys
import types
from fractions import Fraction
from pathlib import Path

import numpy as np

REF = os.environ.get("SUMPY_REFERENCE")
OUT = Path(__file__).with_name("laplace3d_operators.json")

_PLACEHOLDER_PACKAGES = {
    "pytools", "pymbolic", "loopy", "pyopencl", "arraycontext", "boxtree",
    "constantdict", "namedisl", "islpy", "pyvkfft",
}


# {{{ placeholder modules

class _InertMeta(type):
    """Metaclass of inert placeholder classes.

    Calling a placeholder with a single class returns that class (so it works
    as a class decorator); any other call returns a fresh placeholder.
    Subscripting returns the placeholder itself (generic aliases).
    """

    def __call__(cls, *args, **kwargs):
        if cls.__dict__.get("_inert"):
            if len(args) == 1 and not kwargs and isinstance(args[0], type):
                return args[0]
            return _inert("call")
        return super().__call__(*args, **kwargs)

    def __getitem__(cls, item):
        return cls

    def __getattr__(cls, name):
        if name.startswith("__"):
            raise AttributeError(name)
        return _inert(name)


def _inert(name):
    return _InertMeta(name, (), {"_inert": True})


class _PlaceholderModule(types.ModuleType):
    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        value = _inert(name)
        setattr(self, name, value)
        return value


class _PlaceholderFinder(importlib.abc.MetaPathFinder, importlib.abc.Loader):
    def find_spec(self, fullname, path, target=None):
        if fullname.split(".")[0] in _PLACEHOLDER_PACKAGES:
            return importlib.machinery.ModuleSpec(fullname, self, is_package=True)
        return None

    def create_module(self, spec):
        mod = _PlaceholderModule(spec.name)
        mod.__path__ = []
        return mod

    def exec_module(self, module):
        pass


def _install_placeholders():
    sys.meta_path.insert(0, _PlaceholderFinder())
    import functools

    import constantdict as cd_mod
    import pytools

    def memoize_method(f):
        key = "_golden_memo_" + f.__name__

        @functools.wraps(f)
        def wrapper(self, *args, **kwargs):
            cache = self.__dict__.setdefault(key, {})
            k = (args, tuple(sorted(kwargs.items())))
            if k not in cache:
                cache[k] = f(self, *args, **kwargs)
            return cache[k]
        return wrapper

    def memoize(f=None, **_kw):
        def deco(g):
            return functools.lru_cache(maxsize=None)(g)
        return deco(f) if f is not None else deco

    def single_valued(iterable):
        items = list(iterable)
        assert all(x == items[0] for x in items)
        return items[0]

    def tuples_summing_to_at_most(n, length):
        return [t for t in itertools.product(range(n + 1), repeat=length)
                if sum(t) <= n]

    def tuples_below(n, length=None):
        if length is None:
            return list(itertools.product(*[range(k) for k in n]))
        return list(itertools.product(range(n), repeat=length))

    class ProcessLogger:
        def __init__(self, *args, **kwargs):
            pass

        def done(self, *args, **kwargs):
            pass

    class constantdict(dict):  # noqa: N801
        def __hash__(self):
            return hash(frozenset(self.items()))

    pytools.memoize_method = memoize_method
    pytools.memoize = memoize
    pytools.single_valued = single_valued
    pytools.generate_nonnegative_integer_tuples_summing_to_at_most = \
        tuples_summing_to_at_most
    pytools.generate_nonnegative_integer_tuples_below = tuples_below
    pytools.ProcessLogger = ProcessLogger
    cd_mod.constantdict = constantdict

    pkg = types.ModuleType("sumpy")
    pkg.__path__ = [os.path.join(REF, "sumpy")]
    sys.modules["sumpy"] = pkg

# }}}


def _kernels():
    import sympy

    import sumpy.kernel as kernel_mod

    class Laplace3D(kernel_mod.LaplaceKernel):
        def __init__(self):
            object.__setattr__(self, "dim", 3)
            object.__setattr__(self, "expression", "laplace3d")
            object.__setattr__(self, "global_scaling_const", "1/(4pi)")

        def get_expression(self, dvec):
            return 1 / sympy.sqrt(sum(d**2 for d in dvec))

        def __hash__(self):
            return hash("laplace3d-golden")

        def __eq__(self, other):
            return isinstance(other, Laplace3D)

    class Helmholtz3D(kernel_mod.HelmholtzKernel):
        """sumpy's HelmholtzKernel(3) with the wave number fixed at HELM_K;
        get_derivative_taker (HelmholtzDerivativeTaker) and
        get_pde_as_diff_op (Laplacian + k^2, symbol ``k``) are sumpy's."""

        def __init__(self):
            object.__setattr__(self, "dim", 3)
            object.__setattr__(self, "expression", "helmholtz3d")
            object.__setattr__(self, "global_scaling_const", "1/(4pi)")
            object.__setattr__(self, "helmholtz_k_name", "k")
            object.__setattr__(self, "allow_evanescent", False)

        def get_expression(self, dvec):
            r = sympy.sqrt(sum(d**2 for d in dvec))
            return sympy.exp(sympy.I * HELM_K * r) / r

        def __hash__(self):
            return hash("helmholtz3d-golden")

        def __eq__(self, other):
            return isinstance(other, Helmholtz3D)

    return Laplace3D(), Helmholtz3D()


HELM_K = None   # set in main (a sympy Rational)


def generate(knl, orders, out_path, label, complex_valued, extra_subs):
    import sympy

    import sumpy.expansion.local as local_mod
    import sumpy.expansion.m2l as m2l_mod
    import sumpy.expansion.multipole as mpole_mod

    rng = np.random.default_rng(2024)

    def exact(x):
        return sympy.Rational(Fraction(float(x)))

    def ev(expr, subs):
        v = complex(sympy.N(sympy.sympify(expr).doit().xreplace(subs), 40))
        return [v.real, v.imag] if complex_valued else v.real

    vec_syms = sympy.Matrix(sympy.symbols("v0:3"))
    r_src, r_tgt = sympy.symbols("rsrc rtgt")

    cases = []
    for order in orders:
        mpole = mpole_mod.LinearPDEConformingVolumeTaylorMultipoleExpansion(
            knl, order, use_rscale=True)
        local = local_mod.LinearPDEConformingVolumeTaylorLocalExpansion(
            knl, order, use_rscale=True,
            m2l_translation_override=m2l_mod.VolumeTaylorM2LTranslation())
        n = len(mpole)
        ids = [list(mi) for mi in mpole.get_coefficient_identifiers()]
        full_ids = [list(mi) for mi in mpole.get_full_coefficient_identifiers()]
        coeff_syms = list(sympy.symbols(f"c0:{n}"))

        # fixed inputs, exactly representable in binary64
        rs = 0.3125
        rt = 0.625
        a = rng.uniform(-0.15, 0.15, 3).round(6)       # center - source
        b = rng.uniform(-0.15, 0.15, 3).round(6)       # target - center
        d_mm = np.array([0.15625, -0.15625, 0.15625])  # parent - child
        d_ll = -d_mm                                   # child - parent
        d_ml = np.array([1.25, -0.625, 1.875])          # tgt center - src center
        far = rng.uniform(-1, 1, 3).round(6) + np.array([2.0, 0.0, 0.0])
        cin = rng.standard_normal(n).round(8)

        def vsubs(v, extra=()):
            s = {vec_syms[i]: exact(v[i]) for i in range(3)}
            s.update({r_src: exact(rs), r_tgt: exact(rt)})
            s.update({coeff_syms[i]: exact(cin[i]) for i in range(n)})
            s.update(extra_subs)
            s.update(dict(extra))
            return s

        case = {"order": order, "ncoeff": n, "stored_ids": ids,
                "full_ids": full_ids, "rscale_src": rs, "rscale_tgt": rt,
                "coeffs_in": cin.tolist()}

        # P2M / P2L: unit strength source, rscale = rs
        p2m = mpole.coefficients_from_source(knl, vec_syms, None, r_src)
        case["p2m"] = {"avec": a.tolist(),
                       "out": [ev(e, vsubs(a)) for e in p2m]}
        p2l_a = far
        p2l = local.coefficients_from_source(knl, vec_syms, None, r_src)
        case["p2l"] = {"avec": p2l_a.tolist(),
                       "out": [ev(e, vsubs(p2l_a)) for e in p2l]}

        # L2P / M2P: evaluate coeffs_in at bvec, rscale = rs
        l2p = local.evaluate(knl, coeff_syms, vec_syms, r_src)
        case["l2p"] = {"bvec": b.tolist(), "out": ev(l2p, vsubs(b))}
        m2p = mpole.evaluate(knl, coeff_syms, vec_syms, r_src)
        case["m2p"] = {"bvec": far.tolist(), "out": ev(m2p, vsubs(far))}

        # M2M: child (rs) -> parent (rt)
        m2m = mpole.translate_from(mpole, coeff_syms, r_src, vec_syms, r_tgt)
        case["m2m"] = {"dvec": d_mm.tolist(),
                       "out": [ev(e, vsubs(d_mm)) for e in m2m]}
        # L2L: parent (rt) -> child (rs)
        l2l = local.translate_from(local, coeff_syms, r_tgt, vec_syms, r_src)
        case["l2l"] = {"dvec": d_ll.tolist(),
                       "out": [ev(e, vsubs(d_ll)) for e in l2l]}
        # M2L: same rscale on both sides (one tree level), and a mixed case
        m2l = local.translate_from(mpole, coeff_syms, r_src, vec_syms, r_src)
        case["m2l"] = {"dvec": d_ml.tolist(),
                       "out": [ev(e, vsubs(d_ml)) for e in m2l]}
        m2l2 = local.translate_from(mpole, coeff_syms, r_src, vec_syms, r_tgt)
        case["m2l_ratio"] = {"dvec": d_ml.tolist(),
                             "out": [ev(e, vsubs(d_ml)) for e in m2l2]}
        cases.append(case)
        print(f"{label} order {order}: n={n} done", flush=True)

    return {
        "generator": "tests/golden/make_golden.py",
        "expansions": "LinearPDEConformingVolumeTaylor{Multipole,Local}Expansion",
        "conventions": {"avec": "center - source", "bvec": "target - center",
                        "dvec": "target center - source center"},
        "cases": cases}


QBX_OUT_NAME = "qbx3d_pairs.json"


def generate_qbx(lap, helm, line_orders, volume_orders, helm_line_orders,
                 helm_volume_orders):
    """Golden values of the QBX pair expression: sumpy's
    ``LayerPotentialBase._expand`` / ``_evaluate`` (sumpy/qbx.py:113-146) on
    symbolic a (center - source) and b (target - center), evaluated at fixed
    inputs with 40-digit arithmetic, for value, target-, source- and
    directional source-derivative kernels and the line / volume /
    PDE-compressed local expansions."""
    import sympy

    import sumpy.expansion.local as local_mod
    import sumpy.kernel as kernel_mod

    rng = np.random.default_rng(77)

    def exact(x):
        return sympy.Rational(Fraction(float(x)))

    avec = sympy.Matrix(sympy.symbols("a0:3"))
    bvec = sympy.Matrix(sympy.symbols("b0:3"))
    rscale = sympy.Symbol("rscale")
    dir_name = "dsd"

    def pairs_for(knl):
        return [
            ("value", knl, knl, None),
            ("tgt_deriv_1", kernel_mod.AxisTargetDerivative(1, knl), knl, 1),
            ("src_deriv_2", knl, kernel_mod.AxisSourceDerivative(2, knl), 2),
            ("dir_src_deriv", knl, kernel_mod.DirectionalSourceDerivative(knl, dir_name),
             None),
        ]

    expansions = {
        "line": lambda knl, p: local_mod.LineTaylorLocalExpansion(knl, p),
        "volume": lambda knl, p: local_mod.VolumeTaylorLocalExpansion(knl, p),
        "compressed": lambda knl, p: local_mod.LinearPDEConformingVolumeTaylorLocalExpansion(
            knl, p),
    }
    plan = []
    for knl, label, lo, vo, extra in ((lap, "laplace", line_orders, volume_orders, {}),
                                      (helm, "helmholtz", helm_line_orders,
                                       helm_volume_orders,
                                       {sympy.Symbol("k"): HELM_K})):
        for kind in ("line", "volume", "compressed"):
            for p in (lo if kind == "line" else vo):
                plan.append((knl, label, kind, p, extra))

    cases = []
    for knl, label, kind, order, extra in plan:
        expn = expansions[kind](knl, order)
        a = rng.uniform(-0.6, 0.6, 3).round(6) + np.array([0.0, 0.0, 1.0])
        b = rng.uniform(-0.2, 0.2, 3).round(6)
        dvec = rng.standard_normal(3)
        dvec = (dvec / np.linalg.norm(dvec)).round(6)
        subs = {avec[i]: exact(a[i]) for i in range(3)}
        subs.update({bvec[i]: exact(b[i]) for i in range(3)})
        subs.update({sympy.Symbol(f"{dir_name}{i}"): exact(dvec[i]) for i in range(3)})
        subs[rscale] = exact(0.375)
        subs.update(extra)
        for name, tgt_knl, src_knl, _axis in pairs_for(knl):
            coeffs = expn.coefficients_from_source_vec(
                [src_knl], avec, bvec, rscale, weights=[1])
            if kind == "line":
                coeffs = [tgt_knl.postprocess_at_target(c, avec) for c in coeffs]
            csyms = list(sympy.symbols(f"q0:{len(coeffs)}"))
            cvals = {s: sympy.N(sympy.sympify(c).doit().xreplace(subs), 40)
                     for s, c in zip(csyms, coeffs)}
            res = expn.evaluate(tgt_knl, csyms, bvec, rscale)
            v = complex(sympy.N(sympy.sympify(res).doit().xreplace(cvals).xreplace(subs), 40))
            cases.append({"kernel": label, "expansion": kind, "order": order, "pair": name,
                          "avec": a.tolist(), "bvec": b.tolist(), "dir": dvec.tolist(),
                          "value": [v.real, v.imag]})
        print(f"qbx {label} {kind} order {order} done", flush=True)
    return {
        "generator": "tests/golden/make_golden.py --which qbx",
        "conventions": {"avec": "center - source", "bvec": "target - center",
                        "dir": "source derivative direction (DirectionalSourceDerivative)",
                        "value": "pair expression without the kernel scaling, [re, im]"},
        "pairs": {"value": "target and source kernel = base kernel",
                  "tgt_deriv_1": "AxisTargetDerivative(1, base) / base",
                  "src_deriv_2": "base / AxisSourceDerivative(2, base)",
                  "dir_src_deriv": "base / DirectionalSourceDerivative(base)"},
        "k": float(HELM_K),
        "cases": cases}


def main():
    import argparse
    global HELM_K
    ap = argparse.ArgumentParser()
    ap.add_argument("--which", nargs="+", default=["laplace", "helmholtz"],
                    choices=["laplace", "helmholtz", "qbx"])
    ap.add_argument("--laplace-orders", nargs="+", type=int, default=[2, 3, 4, 5, 6, 8])
    ap.add_argument("--helmholtz-orders", nargs="+", type=int, default=[2, 3, 4])
    ap.add_argument("--qbx-line-orders", nargs="+", type=int, default=[3, 5, 8])
    ap.add_argument("--qbx-volume-orders", nargs="+", type=int, default=[3, 5])
    ap.add_argument("--qbx-helmholtz-line-orders", nargs="+", type=int, default=[3, 5])
    ap.add_argument("--qbx-helmholtz-volume-orders", nargs="+", type=int, default=[3])
    ap.add_argument("--out-dir", default=None,
                    help="write the JSON files here instead of next to this script")
    args = ap.parse_args()
    out_lap = OUT if args.out_dir is None else Path(args.out_dir) / OUT.name
    if not REF:
        sys.exit("set SUMPY_REFERENCE to the root of a sumpy source tree")
    _install_placeholders()
    import sympy
    HELM_K = sympy.Rational(5, 2)
    lap, helm = _kernels()
    if "laplace" in args.which:
        data = generate(lap, tuple(args.laplace_orders), out_lap, "laplace", False, {})
        data["kernel"] = "LaplaceKernel(3), expression 1/|d| (scaling applied on output)"
        out_lap.write_text(json.dumps(data, indent=1))
        print("wrote", out_lap)
    if "helmholtz" in args.which:
        out = out_lap.with_name("helmholtz3d_operators.json")
        data = generate(helm, tuple(args.helmholtz_orders), out, "helmholtz", True,
                        {sympy.Symbol("k"): HELM_K})
        data["kernel"] = ("HelmholtzKernel(3), expression exp(i k |d|)/|d| with k = 5/2 "
                          "(scaling applied on output); complex values as [re, im]")
        data["k"] = float(HELM_K)
        out.write_text(json.dumps(data, indent=1))
        print("wrote", out)
    if "qbx" in args.which:
        out = out_lap.with_name(QBX_OUT_NAME)
        data = generate_qbx(lap, helm, args.qbx_line_orders, args.qbx_volume_orders,
                            args.qbx_helmholtz_line_orders, args.qbx_helmholtz_volume_orders)
        out.write_text(json.dumps(data, indent=1))
        print("wrote", out)


if __name__ == "__main__":
    main()
