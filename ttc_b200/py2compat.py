"""Runs modules of the TTC sources (Python 2) under Python 3.

Copies the requested files from a TTC checkout into a scratch directory, expands tabs (the sources
mix tabs and spaces), and rewrites the Python 2 constructs they use: print statements, integer `/`,
`dict.has_key`, list-returning `range`, implicit relative imports, byte-string subprocess output.
The command line uses it to hand `--architecture=avx|avx512|knc|power` requests to TTC's own CPU
code generator (ttc_b200.cpu_delegate); the build recipes of the CPU and GPU reference arms and the
golden fixtures (oracle/make_ref.py, oracle/make_ref_gpu.py, tests/golden/make_golden.py) use it to
drive TTC's generators. Nothing on the GPU path reads the TTC sources.
"""
from __future__ import annotations

import ast
import importlib.util
import io
import shutil
import sys
import tempfile
import tokenize
from pathlib import Path

HELPER = "def _py2div(a, b):\n    return a // b if isinstance(a, int) and isinstance(b, int) else a / b\n"


def _print_statements(src: str) -> str:
    """`print x, y` -> `print(x, y)`; a trailing comma becomes end=' '."""
    toks = list(tokenize.generate_tokens(io.StringIO(src).readline))
    lines = src.splitlines(keepends=True)
    starts = [0]
    for ln in lines:
        starts.append(starts[-1] + len(ln))

    def pos(rc):
        return starts[rc[0] - 1] + rc[1]

    edits = []
    at_stmt_start = True
    for i, t in enumerate(toks):
        if t.type == tokenize.NAME and t.string == "print" and at_stmt_start:
            nxt = toks[i + 1]
            if not (nxt.type == tokenize.OP and nxt.string == "("):
                j = i + 1
                while toks[j].type not in (tokenize.NEWLINE, tokenize.ENDMARKER):
                    j += 1
                k = j - 1
                while toks[k].type in (tokenize.COMMENT, tokenize.NL):
                    k -= 1
                trailing = toks[k].type == tokenize.OP and toks[k].string == ","
                a = pos(t.end)
                b = pos(toks[k].start) if trailing else pos(toks[k].end)
                edits.append((a, b, ", end=' '" if trailing else ""))
        if t.type in (tokenize.NEWLINE, tokenize.INDENT, tokenize.DEDENT):
            at_stmt_start = True
        elif t.type not in (tokenize.NL, tokenize.COMMENT):
            at_stmt_start = False
    for a, b, extra in sorted(edits, reverse=True):
        src = src[:a] + "(" + src[a:b].strip() + extra + ")" + src[b:]
    return src


class _Py2Semantics(ast.NodeTransformer):
    def visit_BinOp(self, node):
        self.generic_visit(node)
        if isinstance(node.op, ast.Div):
            return ast.copy_location(ast.Call(ast.Name("_py2div", ast.Load()), [node.left, node.right], []), node)
        return node

    def visit_AugAssign(self, node):
        self.generic_visit(node)
        if isinstance(node.op, ast.Div):
            target_load = ast.parse(ast.unparse(node.target), mode="eval").body
            call = ast.Call(ast.Name("_py2div", ast.Load()), [target_load, node.value], [])
            return ast.copy_location(ast.Assign([node.target], call), node)
        return node

    def visit_Call(self, node):
        self.generic_visit(node)
        if isinstance(node.func, ast.Attribute) and node.func.attr == "has_key":
            return ast.copy_location(ast.Compare(node.args[0], [ast.In()], [node.func.value]), node)
        if isinstance(node.func, ast.Name) and node.func.id == "range":
            return ast.copy_location(ast.Call(ast.Name("list", ast.Load()), [node], []), node)
        return node


def convert(src: str) -> str:
    src = src.expandtabs(8)
    src = _print_statements(src)
    tree = ast.fix_missing_locations(_Py2Semantics().visit(ast.parse(src)))
    return HELPER + ast.unparse(tree) + "\n"


def convert_tree(src_dir: Path, dst_dir: Path, package_names: list[str]) -> None:
    """Converts every module of a TTC checkout into dst_dir as a Python 3 package."""
    dst_dir.mkdir(parents=True, exist_ok=True)
    for f in src_dir.iterdir():
        if f.is_dir():
            shutil.copytree(f, dst_dir / f.name, dirs_exist_ok=True)
        elif f.suffix != ".py":
            shutil.copy(f, dst_dir / f.name)
    for f in src_dir.glob("*.py"):
        out = convert(f.read_text())
        for other in package_names:
            out = out.replace(f"\nimport {other} as ", f"\nfrom . import {other} as ")
            out = out.replace(f"\nimport {other}\n", f"\nfrom . import {other}\n")
        out = out.replace(".communicate()[0]", ".communicate()[0].decode()")
        out = out.replace("proc = subprocess.Popen(['./transpose.exe'], stderr=subprocess.STDOUT, "
                          "stdout=subprocess.PIPE, env=my_env)",
                          "proc = subprocess.Popen(['./transpose.exe'], stderr=subprocess.STDOUT, "
                          "stdout=subprocess.PIPE, env=my_env, text=True)")
        (dst_dir / f.name).write_text(out)


def load(ttc_dir: Path, names: list[str], package: str = "ttc_ref_py3"):
    """Converts and imports TTC modules (e.g. ["ttc_util", "GPUreference"]) as one package."""
    work = Path(tempfile.mkdtemp(prefix="ttc_py3_"))
    pkg = work / package
    pkg.mkdir()
    (pkg / "__init__.py").write_text("")
    for name in names:
        src = (ttc_dir / f"{name}.py").read_text()
        out = convert(src)
        for other in names:
            out = out.replace(f"\nimport {other}\n", f"\nfrom . import {other}\n")
        (pkg / f"{name}.py").write_text(out)
    sys.path.insert(0, str(work))
    mods = {}
    for name in names:
        mods[name] = importlib.import_module(f"{package}.{name}")
    return mods, work


def cleanup(work: Path):
    shutil.rmtree(work, ignore_errors=True)
