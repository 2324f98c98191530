"""bench.py on a host without a GPU: no name is used before its local import
binds it (the GPU arm cannot run here), and the reference arm (the CPU
pipeline on all host threads) prints one JSON line with the contract's keys."""
import ast
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_no_name_is_used_before_its_local_import():
    tree = ast.parse(open(os.path.join(ROOT, "bench.py")).read())
    problems = []
    for fn in [n for n in ast.walk(tree) if isinstance(n, ast.FunctionDef)]:
        bound = {}
        for node in ast.walk(fn):
            if isinstance(node, (ast.Import, ast.ImportFrom)):
                for alias in node.names:
                    bound.setdefault((alias.asname or alias.name).split(".")[0], node.lineno)
        for node in ast.walk(fn):
            if isinstance(node, ast.Name) and node.id in bound and node.lineno < bound[node.id]:
                problems.append((fn.name, node.id, node.lineno))
    assert problems == []


def test_the_reference_arm_prints_its_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "0"], capture_output=True, text=True,
                         timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "pairs/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
    assert line["higher_is_better"] is True
