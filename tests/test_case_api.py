"""The API surface of the reference's case scripts exists in this package.

``tests/golden/case_api.json`` (made by ``make_case_api.py`` from the
reference's ``cases/*.py``) lists every name the cases import from
curved_lbm, every attribute they read through a module alias, every
attribute they use on a solver object and the keyword arguments of their
calls.  Each must resolve here with the same spelling: an import, a
module attribute, a solver class attribute or an attribute the solver's
constructor assigns, and a keyword the callee's signature accepts.
CPU only: nothing is constructed on a device.
"""

from __future__ import annotations

import ast
import importlib
import inspect
import json

import pytest

from conftest import GOLDEN

API = json.loads((GOLDEN / "case_api.json").read_text())

SOLVER_CLASSES = (("curved_lbm.two_d.curved_boundary_warp", "WarpCurvedBoundaryLBM2D"),
                  ("curved_lbm.three_d.curved_boundary_warp3d", "WarpCurvedBoundaryLBM3D"),
                  ("curved_lbm.three_d.curved_boundary_warp3d", "WarpSparseCurvedBoundaryLBM3D"))
# used by every case driver on every solver, whatever its dimension
COMMON = ("time", "steps", "dt", "dx", "geometry", "material", "boundary_reconstruction_name",
          "initialize_identity", "initialize_from_numpy", "step", "run_until", "refresh_current",
          "active_mask", "system_state", "displacement", "deformation_gradient",
          "deformation_jacobian", "invalid_state", "save_npz", "summary", "numpy_field")


def _instance_attrs(cls) -> set:
    """Names assigned as self.<name> anywhere in the class body, plus class attributes."""
    names = set(dir(cls))
    tree = ast.parse(inspect.getsource(inspect.getmodule(cls)))
    for node in ast.walk(tree):
        if isinstance(node, ast.ClassDef) and node.name == cls.__name__:
            for sub in ast.walk(node):
                if isinstance(sub, ast.Attribute) and isinstance(sub.value, ast.Name) \
                        and sub.value.id == "self" and isinstance(sub.ctx, ast.Store):
                    names.add(sub.attr)
    return names


def _solver_classes():
    return [getattr(importlib.import_module(m), n) for m, n in SOLVER_CLASSES]


@pytest.mark.parametrize("mod,name", [tuple(x) for x in API["imports"] + API["module_attrs"]])
def test_case_imports_resolve(mod, name):
    assert hasattr(importlib.import_module(mod), name), f"{mod}.{name}"


def test_case_solver_attributes_exist():
    per_class = [_instance_attrs(c) for c in _solver_classes()]
    missing = [a for a in API["solver_attrs"] if not any(a in s for s in per_class)]
    assert not missing, missing
    for cls, attrs in zip(_solver_classes(), per_class):
        absent = [a for a in COMMON if a not in attrs]
        assert not absent, (cls.__name__, absent)


def _callee(mod, qual):
    if mod == "<solver>":
        return None
    obj = importlib.import_module(mod)
    for part in qual.split("."):
        obj = getattr(obj, part)
    return obj


def _accepts(fn, keywords) -> bool:
    sig = inspect.signature(fn)
    if any(p.kind is p.VAR_KEYWORD for p in sig.parameters.values()):
        return True
    return all(k in sig.parameters for k in keywords)


@pytest.mark.parametrize("mod,qual,keywords", [tuple(x) for x in API["call_keywords"]],
                         ids=[f"{x[0].split('.')[-1]}:{x[1]}" for x in API["call_keywords"]])
def test_case_call_keywords_accepted(mod, qual, keywords):
    if mod == "<solver>":
        # the scan does not know a call's dimension: some solver class must take them
        targets = [getattr(c, qual) for c in _solver_classes() if hasattr(c, qual)]
        assert targets and any(_accepts(fn, keywords) for fn in targets), (qual, keywords)
    else:
        fn = _callee(mod, qual)
        assert _accepts(fn, keywords), (qual, [k for k in keywords
                                               if k not in inspect.signature(fn).parameters])
