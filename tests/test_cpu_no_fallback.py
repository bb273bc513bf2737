"""The product path has no fallback: without its CUDA library it raises, and the package
never imports the oracle (the oracle is test infrastructure)."""
import ast
import glob
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_missing_library_raises():
    code = (
        "from snowsimulation_b200 import _native\n"
        "try:\n"
        "    _native.load('/nonexistent/libsnowb200.so')\n"
        "except _native.SnowError as e:\n"
        "    print('raised', e)\n"
        "else:\n"
        "    print('loaded')\n"
    )
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert out.stdout.startswith("raised"), out.stdout


def test_package_does_not_import_the_oracle():
    for path in glob.glob(os.path.join(ROOT, "snowsimulation_b200", "*.py")):
        tree = ast.parse(open(path).read())
        for node in ast.walk(tree):
            if isinstance(node, ast.Import):
                names = [a.name for a in node.names]
            elif isinstance(node, ast.ImportFrom):
                names = [node.module or ""]
            else:
                continue
            assert not any(n == "oracle" or n.startswith("oracle.") for n in names), (path, names)
