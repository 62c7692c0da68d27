"""The C++ drop-in boundary: the reference's own example programs compile,
unmodified, against this library's headers at the reference's include paths
(include/xfdtd/...) with the shipped xtensor subset (include/xtensor_subset),
and the two the GPU tests run are linked against libxfdtd_host.so."""
import os
import subprocess

import pytest

from tests import examples_build as X

pytestmark = pytest.mark.skipif(not X.available(),
                                reason="the reference's example sources are not present")


@pytest.mark.parametrize("name", sorted(X.EXAMPLES))
def test_reference_example_compiles_unmodified(name):
    src = os.path.join(X.example_dir(), X.EXAMPLES[name])
    r = subprocess.run(X.compile_cmd(src, None), capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]


def test_linked_examples_resolve_this_library():
    for path in X.build():
        assert os.access(path, os.X_OK)
        out = subprocess.run(["ldd", path], capture_output=True, text=True).stdout
        for lib in ("libxfdtd_host.so", "libxfd_engine.so"):
            line = next(l for l in out.splitlines() if lib in l)
            assert "not found" not in line and os.path.realpath(X.LIBDIR) in \
                os.path.realpath(line.split("=>")[1].split("(")[0].strip())
