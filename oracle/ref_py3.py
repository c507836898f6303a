"""ORACLE -- test infrastructure only (used to produce golden fixtures).

Imports the reference's own generator (TCCG, Python 2) under Python 3 so
that its parser, index fusion, classification and emitted loop-nest
reference can be run here and their outputs frozen as fixtures under
tests/golden/. The reference sources are read from the read-only reference
checkout and converted in memory; the converted modules are written only to
oracle/_ref/py3/ (git-ignored, never committed).

The conversion is mechanical and semantic-preserving for the code paths used:

* tabs expanded to 8 columns (Python 2's rule);
* ``print`` statements become ``print(...)`` calls (a trailing comma becomes
  ``end=" "``), found with the tokenizer so strings are never touched;
* every ``/`` becomes ``_py2div(a, b)``, which floors when both operands are
  integers, exactly like Python 2 (``/=`` likewise);
* ``d.has_key(k)`` becomes ``k in d``; ``d.keys()[i]`` becomes
  ``list(d.keys())[i]``;
* ``min``/``max`` keep Python 2's cross-type order (numbers before lists,
  e.g. ``min(8, strategies)`` is 8, tccg/gett.py:792).

Usage: ``load_reference(ref_root)`` returns a dict of the converted modules.
"""
from __future__ import annotations

import ast
import io
import os
import sys
import tokenize
from typing import Dict

# The reference checkout: $TCCG_REFERENCE_ROOT, else a directory named
# "reference" beside the repository; where neither exists the reference-built
# checkers are skipped (the committed fixtures and prebuilt files are used).
DEFAULT_REF = os.environ.get("TCCG_REFERENCE_ROOT") or os.path.join(
    os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))), "reference")
_HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(_HERE, "_ref", "py3")

MODULES = ["Index", "register", "instructions", "arch", "tensor", "tccg_util",
           "transpose", "ttgemmt", "gemm_loop", "gett", "sql_util", "tccg"]

_PRELUDE = '''
def _py2div(a, b):
    if isinstance(a, int) and isinstance(b, int):
        return a // b
    return a / b

def _py2order(x):
    # Python 2 orders numbers before every other type
    return (0, x) if isinstance(x, (int, float)) else (1, 0)

def _py2min(*args, **kw):
    try:
        return min(*args, **kw)
    except TypeError:
        items = args[0] if len(args) == 1 else args
        return sorted(items, key=_py2order)[0]

def _py2max(*args, **kw):
    try:
        return max(*args, **kw)
    except TypeError:
        items = args[0] if len(args) == 1 else args
        return sorted(items, key=_py2order)[-1]
'''


def _convert_prints(src: str) -> str:
    """Rewrite Python-2 print statements into calls, using token positions."""
    lines = src.splitlines(keepends=True)
    toks = list(tokenize.generate_tokens(io.StringIO(src).readline))
    edits = []  # (start(row,col), end(row,col), replacement-for-args, trailing_comma)
    at_stmt_start = True
    i = 0
    while i < len(toks):
        t = toks[i]
        if t.type in (tokenize.NEWLINE, tokenize.INDENT, tokenize.DEDENT, tokenize.NL,
                      tokenize.COMMENT):
            if t.type in (tokenize.NEWLINE, tokenize.INDENT, tokenize.DEDENT):
                at_stmt_start = True
            i += 1
            continue
        if at_stmt_start and t.type == tokenize.NAME and t.string == "print":
            nxt = toks[i + 1]
            # find the end of the logical line
            j = i + 1
            depth = 0
            while toks[j].type != tokenize.NEWLINE and toks[j].type != tokenize.ENDMARKER:
                if toks[j].type == tokenize.OP and toks[j].string in "([{":
                    depth += 1
                elif toks[j].type == tokenize.OP and toks[j].string in ")]}":
                    depth -= 1
                if toks[j].type == tokenize.OP and toks[j].string == ";" and depth == 0:
                    break
                j += 1
            last = j - 1
            while toks[last].type in (tokenize.COMMENT, tokenize.NL):
                last -= 1
            trailing = toks[last].type == tokenize.OP and toks[last].string == ","
            if nxt.type == tokenize.NEWLINE or (nxt.type == tokenize.OP and nxt.string == ";"):
                edits.append((t.end, t.end, "()", False, None))
            else:
                start = nxt.start
                end = toks[last].start if trailing else toks[last].end
                edits.append((start, end, None, trailing, toks[last].end if trailing else None))
            i = j
            at_stmt_start = False
            continue
        at_stmt_start = False
        i += 1

    # apply edits bottom-up on absolute offsets
    offs = [0]
    for ln in lines:
        offs.append(offs[-1] + len(ln))
    ab = lambda rc: offs[rc[0] - 1] + rc[1]
    out = src
    for (s, e, repl, trailing, tend) in sorted(edits, key=lambda x: ab(x[0]), reverse=True):
        if repl is not None:
            out = out[:ab(s)] + repl + out[ab(e):]
        else:
            body = out[ab(s):ab(e)]
            stop = ab(tend) if trailing else ab(e)
            tail = ', end=" ")' if trailing else ")"
            out = out[:ab(s)] + "(" + body + tail + out[stop:]
    return out


class _Py2Semantics(ast.NodeTransformer):
    def visit_BinOp(self, node):
        self.generic_visit(node)
        if isinstance(node.op, ast.Div):
            return ast.copy_location(
                ast.Call(func=ast.Name("_py2div", ast.Load()), args=[node.left, node.right],
                         keywords=[]), node)
        return node

    def visit_AugAssign(self, node):
        self.generic_visit(node)
        if isinstance(node.op, ast.Div):
            tgt_load = ast.parse(ast.unparse(node.target), mode="eval").body
            return ast.copy_location(
                ast.Assign(targets=[node.target],
                           value=ast.Call(func=ast.Name("_py2div", ast.Load()),
                                          args=[tgt_load, node.value], keywords=[])), node)
        return node

    def visit_Call(self, node):
        self.generic_visit(node)
        f = node.func
        if isinstance(f, ast.Name) and f.id in ("min", "max"):
            node.func = ast.Name("_py2" + f.id, ast.Load())
            return node
        if isinstance(f, ast.Attribute) and f.attr == "has_key" and len(node.args) == 1:
            return ast.copy_location(
                ast.Compare(left=node.args[0], ops=[ast.In()], comparators=[f.value]), node)
        return node

    def visit_Subscript(self, node):
        self.generic_visit(node)
        v = node.value
        if (isinstance(v, ast.Call) and isinstance(v.func, ast.Attribute)
                and v.func.attr in ("keys", "values", "items")):
            node.value = ast.Call(func=ast.Name("list", ast.Load()), args=[v], keywords=[])
        return node


def convert_source(src: str) -> str:
    src = "".join(l.expandtabs(8) for l in src.splitlines(keepends=True))
    src = _convert_prints(src)
    tree = ast.parse(src)
    tree = _Py2Semantics().visit(tree)
    ast.fix_missing_locations(tree)
    return _PRELUDE + ast.unparse(tree) + "\n"


def convert_reference(ref_root: str = DEFAULT_REF, out_dir: str = OUT_DIR) -> str:
    """Convert the reference's generator modules into ``out_dir``."""
    os.makedirs(out_dir, exist_ok=True)
    for m in MODULES:
        path = os.path.join(ref_root, "tccg", m + ".py")
        with open(path) as f:
            src = f.read()
        with open(os.path.join(out_dir, m + ".py"), "w") as f:
            f.write(convert_source(src))
    return out_dir


def load_reference(ref_root: str = DEFAULT_REF) -> Dict[str, object]:
    """Convert (if needed) and import the reference's modules."""
    out = convert_reference(ref_root)
    if out not in sys.path:
        sys.path.insert(0, out)
    import importlib
    mods = {}
    for m in MODULES:
        mods[m] = importlib.import_module(m)
    return mods


def reference_available(ref_root: str = DEFAULT_REF) -> bool:
    return os.path.isfile(os.path.join(ref_root, "tccg", "tccg.py"))
