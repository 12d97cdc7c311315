"""bench.py's command line: every workload it dispatches to exists (no GPU needed)."""
import ast
import builtins
import os

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_every_function_called_by_main_is_defined():
    tree = ast.parse(open(os.path.join(ROOT, "bench.py")).read())
    main = next(n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == "main")
    called = {n.func.id for n in ast.walk(main) if isinstance(n, ast.Call) and isinstance(n.func, ast.Name)}
    defined = {n.name for n in tree.body if isinstance(n, (ast.FunctionDef, ast.ClassDef))}
    missing = sorted(c for c in called if c not in defined and not hasattr(builtins, c) and not hasattr(bench, c))
    assert not missing, missing
    for name in ("run_large_ns", "run_tracers", "run_ensemble", "run_ours"):
        assert callable(getattr(bench, name)), name
