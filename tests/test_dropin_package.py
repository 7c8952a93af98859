"""The reference's unmodified Python package (``scatrs``) over this repository's binding as its
extension module ``scatrs._scatrs``: it imports (it reads ``__version__`` and the ``MAX_*``
limits at import, python/scatrs/mie.py:49-56, layered.py:60, special.py:19-22, tmatrix.py:45,
__init__.py:81), and the library's failures reach its callers as the classes of
``scatrs.errors`` (scatrs-py/src/errors.rs:14-45), NotConvergedError with achieved/requested.

The package's source is taken from a checkout of the reference beside this repository (or the
directory named by SCATRS_REFERENCE_ROOT); the test is skipped where there is none. It runs in a
subprocess, so that the package's modules do not outlive it. Without a GPU an ensemble call
stops at the device check, which must raise the package's ScatrsError.
"""

import os
import subprocess
import sys
import textwrap

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("SCATRS_REFERENCE_ROOT", os.path.join(os.path.dirname(ROOT), "reference"))
PKG = os.path.join(REF, "python")

pytestmark = pytest.mark.skipif(not os.path.isdir(os.path.join(PKG, "scatrs")),
                                reason="no checkout of the reference's Python package")

SCRIPT = textwrap.dedent("""
    import math, pickle, sys
    sys.path.insert(0, {root!r})
    sys.path.insert(0, {pkg!r})
    import scatrs_b200._scatrs as ours
    sys.modules["scatrs._scatrs"] = ours
    import scatrs
    from scatrs import _scatrs
    assert _scatrs is ours
    assert scatrs.__version__ == "0.3.0", scatrs.__version__
    assert scatrs.mie.MAX_MIE_ORDER == 1 << 20
    assert scatrs.mie.MAX_MIE_VALUES == 1 << 27
    assert scatrs.mie.MAX_GREEK_ORDER == 1 << 21
    assert scatrs.layered.MAX_LAYERS == 16
    assert scatrs.tmatrix.MAX_TMATRIX_ORDER == 500
    assert scatrs.special.MAX_GAUSS_LEGENDRE_POINTS == 1 << 17
    assert scatrs.special.MAX_WIGNER_D_VALUES == 1 << 28

    # The library's error path raises the package's own classes.
    t = _scatrs._testing
    for variant, cls in (("InvalidInput", scatrs.InvalidInputError),
                         ("OutsideValidatedDomain", scatrs.OutsideValidatedDomainError)):
        try:
            t.raise_core_error(variant, "x > 2e4")
        except scatrs.ScatrsError as e:
            assert type(e) is cls, type(e)
            assert "x > 2e4" in str(e)
        else:
            raise AssertionError("no exception")
    try:
        t.raise_core_error("NotConverged", achieved=1e-3, requested=1e-6)
    except scatrs.NotConvergedError as e:
        assert type(e) is scatrs.NotConvergedError
        assert (e.achieved, e.requested) == (1e-3, 1e-6)
        assert isinstance(e, ArithmeticError)
        back = pickle.loads(pickle.dumps(e))
        assert (back.achieved, back.requested) == (1e-3, 1e-6)
    try:
        t.raise_core_error("NotConverged", achieved=math.inf, requested=1e-8)
    except scatrs.NotConvergedError as e:
        assert e.achieved == math.inf and e.requested == 1e-8

    # Parameter names through the package (ensemble_parameters, scatrs-py/src/ensemble.rs:172-188).
    ens = scatrs.Ensemble(scatrs.Sphere(1.45 + 2e-3j), scatrs.LogNormal(0.1, 1.5))
    names = _scatrs.ensemble_parameters(
        [(("lognormal", 0.1, 1.5), ("sphere", None), 1.0)], False)
    assert names == ["median_radius", "width", "m_real", "m_imag"], names

    # The ensemble call itself: on a GPU it computes; without one, the device check raises the
    # package's ScatrsError.
    import numpy as np
    try:
        r = ens.compute(np.array([0.5, 1.0]), greek=8)
        assert r.c_ext.shape == (2,) and np.all(np.isfinite(r.c_ext))
        print("COMPUTED")
    except scatrs.ScatrsError as e:
        assert type(e) is scatrs.ScatrsError, type(e)
        assert "no usable CUDA device" in str(e), str(e)
        print("NO_DEVICE")
    print("DROPIN_OK")
""")


def test_reference_package_imports_and_raises_its_classes():
    out = subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT, pkg=PKG)],
                         capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-3000:]
    assert "DROPIN_OK" in out.stdout
