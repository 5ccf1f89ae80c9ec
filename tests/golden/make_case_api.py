#!/usr/bin/env python3
"""Record the curved_lbm API surface that the reference's case scripts use.

The reference's drivers (``cases/*.py``) are the users this package must
serve unchanged.  This script parses them (``ast``, nothing is executed) and
writes ``case_api.json`` beside it:

* ``imports``: every ``from curved_lbm.<module> import <name>``;
* ``module_attrs``: every ``<alias>.<name>`` read through a module alias
  (``from curved_lbm.three_d import curved_boundary_warp3d as cb`` ...);
* ``solver_attrs``: every attribute read or called on a variable named
  ``solver`` (the cases' name for the solver object);
* ``call_keywords``: for calls of an imported class, of a constructor method
  on it (``Class.method(...)``) or of a solver method, the keyword names
  passed explicitly.

Run where the reference checkout is readable::

    python tests/golden/make_case_api.py --ref <reference checkout>

(or set CVLBM_REFERENCE_ROOT).
"""

from __future__ import annotations

import argparse
import ast
import json
import os
from collections import defaultdict
from pathlib import Path

HERE = Path(__file__).resolve().parent


class _Scan(ast.NodeVisitor):
    def __init__(self):
        self.imports: set = set()
        self.aliases: dict = {}     # alias -> module
        self.names: dict = {}       # imported name -> module
        self.module_attrs: set = set()
        self.solver_attrs: set = set()
        self.keywords: dict = defaultdict(set)

    def visit_ImportFrom(self, node):
        mod = node.module or ""
        if mod.startswith("curved_lbm"):
            for a in node.names:
                sub = f"{mod}.{a.name}"
                if a.name in ("two_d", "three_d") or a.name.endswith(("_warp", "_warp3d",
                                                                      "stencil3d")):
                    self.aliases[a.asname or a.name] = sub
                else:
                    self.imports.add((mod, a.name))
                    self.names[a.asname or a.name] = (mod, a.name)
        self.generic_visit(node)

    def visit_Import(self, node):
        for a in node.names:
            if a.name.startswith("curved_lbm") and a.asname:
                self.aliases[a.asname] = a.name
        self.generic_visit(node)

    def visit_Attribute(self, node):
        if isinstance(node.value, ast.Name):
            base = node.value.id
            if base in self.aliases:
                self.module_attrs.add((self.aliases[base], node.attr))
            elif base == "solver":
                self.solver_attrs.add(node.attr)
        self.generic_visit(node)

    def _callee(self, func):
        """(module, qualified name) of a call target we track, else None."""
        if isinstance(func, ast.Name) and func.id in self.names:
            return self.names[func.id]
        if isinstance(func, ast.Attribute):
            v = func.value
            if isinstance(v, ast.Name):
                if v.id in self.aliases:
                    return (self.aliases[v.id], func.attr)
                if v.id in self.names:
                    mod, name = self.names[v.id]
                    return (mod, f"{name}.{func.attr}")
                if v.id == "solver":
                    return ("<solver>", func.attr)
            if isinstance(v, ast.Attribute) and isinstance(v.value, ast.Name) \
                    and v.value.id in self.aliases:
                return (self.aliases[v.value.id], f"{v.attr}.{func.attr}")
        return None

    def visit_Call(self, node):
        key = self._callee(node.func)
        if key is not None:
            kws = {k.arg for k in node.keywords if k.arg is not None}
            self.keywords[key] |= kws
        self.generic_visit(node)


def scan(cases_dir: Path) -> dict:
    out = {"imports": set(), "module_attrs": set(), "solver_attrs": set(),
           "call_keywords": defaultdict(set), "files": []}
    for path in sorted(cases_dir.glob("*.py")):
        s = _Scan()
        s.visit(ast.parse(path.read_text(), filename=str(path)))
        out["files"].append(path.name)
        out["imports"] |= s.imports
        out["module_attrs"] |= s.module_attrs
        out["solver_attrs"] |= s.solver_attrs
        for k, v in s.keywords.items():
            out["call_keywords"][k] |= v
    return {
        "source": "cases/*.py of the reference checkout (parsed, not executed)",
        "files": out["files"],
        "imports": sorted(list(t) for t in out["imports"]),
        "module_attrs": sorted(list(t) for t in out["module_attrs"]),
        "solver_attrs": sorted(out["solver_attrs"]),
        "call_keywords": sorted([k[0], k[1], sorted(v)] for k, v in out["call_keywords"].items()
                                if v),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("CVLBM_REFERENCE_ROOT"),
                    help="root of the reference checkout (or CVLBM_REFERENCE_ROOT)")
    args = ap.parse_args()
    if not args.ref:
        ap.error("--ref (or CVLBM_REFERENCE_ROOT) is required")
    data = scan(Path(args.ref) / "cases")
    (HERE / "case_api.json").write_text(json.dumps(data, indent=1) + "\n")
    print(f"{len(data['files'])} files, {len(data['imports'])} imports, "
          f"{len(data['module_attrs'])} module attributes, {len(data['solver_attrs'])} solver "
          f"attributes, {len(data['call_keywords'])} call sites with keywords")


if __name__ == "__main__":
    main()
