"""The C-ABI library loads without a GPU, exports every function declared in
include/cloudsc_b200.h, agrees with the Python struct mirror, and reports
argument errors with CLOUDSC's error codes (checked before any device work)."""
import ctypes
import os
import re

import numpy as np
import pytest

from openifs_b200 import cloudsc, fields, inputs
from openifs_b200.params import CloudscParams

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(ROOT, "include", "cloudsc_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(cloudsc_b200_\w+)\s*\(", txt)))


def test_exports_every_declared_symbol(built):
    lib = cloudsc.lib()
    names = _declared()
    assert len(names) >= 9
    for n in names:
        assert hasattr(lib, n), n


def test_struct_size_matches(built):
    assert ctypes.sizeof(CloudscParams) == cloudsc.lib().cloudsc_b200_params_size()


def test_version(built):
    assert b"sm_100a" in cloudsc.lib().cloudsc_b200_version()


def test_error_codes_without_device_work(built):
    p = cloudsc.default_params()
    try:
        cloudsc.setup(p)  # on a CPU-only host this fails at the upload (-4) but keeps p
    except cloudsc.CloudscError as e:
        assert e.code == -4
    arrs = {n: None for n, *_ in fields.BATCHED_FIELDS}
    # a NULL array
    with pytest.raises(cloudsc.CloudscError) as e:
        cloudsc.cloudsc_batched(p, {**arrs, **{n: np.zeros(1) for n in fields.INPUT_NAMES}},
                                32, 137, 2, 64, 3600.0, validate=False)
    assert e.value.code == -1
    full = {n: np.zeros(1) for n, *_ in fields.BATCHED_FIELDS}
    # NGPTOT inconsistent with NPROMA*NGPBLKS
    with pytest.raises(cloudsc.CloudscError) as e:
        cloudsc.cloudsc_batched(p, full, 32, 137, 2, 65, 3600.0, validate=False)
    assert e.value.code == -2
    # KLEV smaller than NCLDTOP
    with pytest.raises(cloudsc.CloudscError) as e:
        cloudsc.cloudsc_batched(p, full, 32, 10, 2, 64, 3600.0, validate=False)
    assert e.value.code == -2
    # parameters that differ from the uploaded ones
    q = p.copy()
    q.ramid = 0.9
    with pytest.raises(cloudsc.CloudscError) as e:
        cloudsc.cloudsc_batched(q, full, 32, 137, 2, 64, 3600.0, validate=False)
    assert e.value.code == -5
    # the Python mirror checks presence, dtype, size and placement first
    with pytest.raises(cloudsc.CloudscError) as e:
        cloudsc.cloudsc_batched(p, full, 32, 137, 2, 64, 3600.0)
    assert e.value.code == -2
    host = fields.alloc(2, 32, 137)
    cloudsc._check_batched(host, 32, 137, 2, device=False)  # the right shapes pass
    bad = dict(host, pt=host["pt"].astype(np.float32))
    with pytest.raises(cloudsc.CloudscError) as e:
        cloudsc._check_batched(bad, 32, 137, 2, device=False)
    assert e.value.code == -2
    with pytest.raises(cloudsc.CloudscError) as e:
        cloudsc._check_batched({k: v for k, v in host.items() if k != "ktype"}, 32, 137, 2, device=False)
    assert e.value.code == -1
    # bad launch shape
    with pytest.raises(cloudsc.CloudscError):
        cloudsc.set_launch(0, 48, 0)


def test_block_entry_argument_checks(built):
    p = cloudsc.default_params()
    try:
        cloudsc.setup(p)
    except cloudsc.CloudscError:
        pass
    with pytest.raises(cloudsc.CloudscError) as e:  # KFDIA > KLON
        cloudsc.cloudsc_block(p, 1, 40, 32, 137, 3600.0, {})
    assert e.value.code == -2
    with pytest.raises(cloudsc.CloudscError) as e:  # missing required arrays
        cloudsc.cloudsc_block(p, 1, 32, 32, 137, 3600.0, {})
    assert e.value.code == -1


def test_bytes_per_column():
    rb, wb = fields.bytes_per_column()
    assert (rb, wb) == (28528, 25328)


def test_gemm_rejects_misaligned_epilogue_arrays(built):
    """cs_conv_gemm checks its arrays before any device work: TMA operands on
    16 bytes, the epilogue's arrays on 32 bytes (its 256-bit accesses);
    anything else returns CS_E_ARG without a launch."""
    import ctypes
    import torch
    from openifs_b200 import tcgemm
    a = torch.zeros(256, 128, dtype=torch.bfloat16)
    w = torch.zeros(1, 128, 128, dtype=torch.bfloat16)
    out = torch.zeros(256 * 128 + 16, dtype=torch.bfloat16)
    fn = tcgemm._lib_fn()

    def call(out_ptr, resid_ptr=None):
        d = tcgemm.GemmDesc(a.data_ptr(), w.data_ptr(), 256, 128, 128, 1, 0, 0, tcgemm.EPI_SILU, None,
                            out_ptr, None, resid_ptr, None, None, None, None)
        return fn(ctypes.byref(d), None)

    base = out.data_ptr()
    assert base % 32 == 0
    assert call(base + 16) == -2            # 16-byte aligned output: rejected
    assert call(base, a.data_ptr() + 16) == -2  # residual off by 16 bytes
    d = tcgemm.GemmDesc(a.data_ptr() + 8, w.data_ptr(), 256, 128, 128, 1, 0, 0, tcgemm.EPI_SILU, None,
                        base, None, None, None, None, None, None)
    assert fn(ctypes.byref(d), None) == -2  # TMA operand off by 8 bytes


def test_post_rejects_misaligned_network_output(built):
    """cs_post reads the network output 16 bytes at a time: an output array
    that is not 16-byte aligned returns CS_E_ARG before any launch."""
    import ctypes
    import torch
    from openifs_b200 import surrogate as S
    p = cloudsc.default_params()
    nproma, nblk = 32, 1
    tdt = lambda dt: torch.float64 if np.dtype(dt) == np.float64 else torch.int32
    dev = fields.alloc(nblk, nproma, S.KLEV, alloc_fn=lambda shape, dt: torch.zeros(shape, dtype=tdt(dt)))
    colsum = torch.zeros(nproma * nblk, S.KLEV, 2)
    c = S.columns(dev, nproma, nblk, colsum, p)
    y = torch.zeros(nproma * nblk * S.LP * 64 + 8)
    assert y.data_ptr() % 16 == 0
    g = S.Guard()
    g.capacity = 0
    nflag = torch.zeros(1, dtype=torch.int32)
    L = S._lib()
    rc = L.cs_post(ctypes.byref(c), y.data_ptr() + 4, 2, ctypes.byref(g), nflag.data_ptr(), None, None, None)
    assert rc == -2
    rc = L.cs_post(ctypes.byref(c), y.data_ptr() + 8, 2, ctypes.byref(g), nflag.data_ptr(), None, None, None)
    assert rc == -2
