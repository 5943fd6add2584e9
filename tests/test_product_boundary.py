"""The package never reaches the CPU oracle or a CPU fallback: no module of
diffswe2d_b200 imports, loads or runs anything under oracle/, and the
native binding refuses to run without its CUDA library."""
import ast
from pathlib import Path

import pytest

PKG = Path(__file__).resolve().parent.parent / "diffswe2d_b200"


def _imports(path: Path):
    tree = ast.parse(path.read_text())
    for node in ast.walk(tree):
        if isinstance(node, ast.Import):
            for a in node.names:
                yield a.name
        elif isinstance(node, ast.ImportFrom):
            yield node.module or ""


@pytest.mark.parametrize("path", sorted(PKG.glob("*.py")), ids=lambda p: p.name)
def test_package_module_does_not_touch_the_oracle(path):
    assert not any(name.split(".")[0] == "oracle" for name in _imports(path))
    text = path.read_text()
    assert "oracle/" not in text and "swe_oracle" not in text


def test_missing_library_raises(tmp_path, monkeypatch):
    from diffswe2d_b200 import _native as nat
    monkeypatch.setattr(nat, "LIB_PATH", tmp_path / "missing.so")
    monkeypatch.setattr(nat, "_lib", None)
    with pytest.raises(nat.NativeLibraryError):
        nat.lib()
