"""bench.py on the CPU: every function it calls by name exists at module level (a workload flag
that dispatches to a missing function would only fail on a GPU box), and the reference arm prints
one JSON line with the contract's keys on a small table."""
import ast
import builtins
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _names_defined(tree):
    out = set(dir(builtins))
    for node in ast.walk(tree):
        if isinstance(node, (ast.FunctionDef, ast.AsyncFunctionDef, ast.ClassDef)):
            out.add(node.name)
            a = node.args if not isinstance(node, ast.ClassDef) else None
            if a is not None:
                for arg in a.args + a.kwonlyargs + a.posonlyargs + [a.vararg, a.kwarg]:
                    if arg is not None:
                        out.add(arg.arg)
        elif isinstance(node, (ast.Import, ast.ImportFrom)):
            for al in node.names:
                out.add((al.asname or al.name).split(".")[0])
        elif isinstance(node, ast.Name) and isinstance(node.ctx, ast.Store):
            out.add(node.id)
        elif isinstance(node, ast.arg):
            out.add(node.arg)
        elif isinstance(node, ast.ExceptHandler) and node.name:
            out.add(node.name)
    return out


def test_every_called_name_is_defined():
    tree = ast.parse((ROOT / "bench.py").read_text())
    defined = _names_defined(tree)
    called = {n.func.id for n in ast.walk(tree) if isinstance(n, ast.Call) and isinstance(n.func, ast.Name)}
    assert called <= defined, sorted(called - defined)


def test_reference_arm_line_on_cpu():
    p = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--cap-log", "16", "--steps", "1",
                        "--warmup", "0", "--no-reference-gpu"], capture_output=True, text=True, timeout=300,
                       cwd=str(ROOT))
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, p.stdout
    r = json.loads(lines[0])
    assert r["impl"] == "reference" and r["unit"] == "Mops/s" and r["value"] > 0
    assert r["e2e"]["h2d_bytes_per_step"] == 0 and r["cpu_baseline"]["kind"] == "port"
    assert r["cpu_baseline"]["inserts_failed"] == 0
