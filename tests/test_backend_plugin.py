"""The B200 backend against the reference's own plugin check.

The reference activates a backend by rewriting the class of its ``bm``
object and checks it with MasterBackend.verify_backend
(blond/utils/bmath_backends.py:203-256): every attribute a backend sets must
be declared by MasterBackend and must not be None.  Here a MasterBackend
subclass takes every attribute of blond_b200.bmath.B200Backend, is
installed into the reference's ``bm`` the reference's way and verified by
the reference's code; and the attribute list blond_b200 restates must be
exactly the reference's.  The reference is imported in a child process
(its import stubs for matplotlib and h5py stay out of this one) and only
where its checkout and oracle/_ref are present; nothing here needs a GPU.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import sys
sys.path.insert(0, {root!r})
sys.path.insert(0, {oracle!r})
import ref_harness
ref_harness.import_reference("double")
from blond.utils import bmath as bm
from blond.utils.bmath_backends import MasterBackend
from blond_b200 import bmath as b200

declared = list(MasterBackend().__dict__)
assert declared == list(b200.MASTER_ATTRIBUTES), (
    sorted(set(declared) ^ set(b200.MASTER_ATTRIBUTES)))


class GpuB200Backend(MasterBackend):
    def __init__(self):
        MasterBackend.__init__(self)
        self.__dict__.update(b200.B200Backend().__dict__)


GpuB200Backend().verify_backend()
bm.__class__ = GpuB200Backend
GpuB200Backend.__init__(bm)
bm.verify_backend()
assert bm.kick is b200.kick and bm.slice_beam is b200.slice_beam
assert bm.linear_interp_kick is b200.linear_interp_kick and bm.device == "GPU_B200"
print("PLUGIN_OK")
"""


def test_backend_passes_the_reference_plugin_check():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_harness
    lib = os.path.join(ROOT, "oracle", "_ref", "libblond_ref_double.so")
    if not (os.path.isdir(os.path.join(ref_harness.DEFAULT_REF, "blond"))
            and os.path.exists(lib)):
        pytest.skip("the reference checkout or oracle/_ref is not present")
    code = CHILD.format(root=ROOT, oracle=os.path.join(ROOT, "oracle"))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and "PLUGIN_OK" in r.stdout, r.stdout + r.stderr


def test_backend_sets_every_declared_attribute():
    from blond_b200.bmath import MASTER_ATTRIBUTES, B200Backend
    b = B200Backend()
    assert set(b.__dict__) == set(MASTER_ATTRIBUTES)
    assert all(v is not None for v in b.__dict__.values())
