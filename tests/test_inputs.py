"""The seeded input generator: per-block determinism and physical ranges."""
import numpy as np
import pytest

from openifs_b200 import cloudsc, fields, inputs


def test_blocks_regenerate_identically(built):
    p = cloudsc.default_params()
    full = inputs.generate(6, 16, p, seed=4)
    part = inputs.generate(6, 16, p, seed=4, blocks=[4, 1])
    for n in fields.INPUT_NAMES:
        assert np.array_equal(part[n][0], full[n][4]), n
        assert np.array_equal(part[n][1], full[n][1]), n
    other = inputs.generate(6, 16, p, seed=5, blocks=[4])
    assert not np.array_equal(other["pt"][0], full["pt"][4])


def test_ranges(built):
    p = cloudsc.default_params()
    a = inputs.generate(8, 64, p, seed=1)
    assert a["paph"][:, 0].max() == 0.0 and np.all(np.diff(a["paph"], axis=1) > 0)
    ps = a["paph"][:, -1]
    assert ps.min() >= 98000.0 and ps.max() <= 103000.0
    assert a["pt"].min() > 200.0 and a["pt"].max() < 320.0
    assert 0.0 <= a["pa"].min() and a["pa"].max() <= 1.0
    assert a["pq"].max() < 0.05 and a["pq"].min() > 0.0
    cl = a["pclv"]
    assert cl.min() >= 0.0 and cl.max() <= 5e-3
    warm = a["pt"] > 273.0
    assert np.all(cl[:, 1][warm] == 0.0) and np.all(cl[:, 3][warm] == 0.0)
    nc = int(p.ncldtop)
    assert np.all(cl[:, :, : nc - 1] == 0.0)
    assert set(np.unique(a["ktype"])) <= {0, 1, 2, 3}
    assert np.all((a["ktype"] > 0) == (a["ldcum"] > 0))
    assert np.all(a["pmfd"] <= 0.0) and np.all(a["pmfu"] >= 0.0)
    assert abs(a["ldcum"].mean() - 0.3) < 0.1


def test_l137_table():
    a, b = inputs.l137_ab()
    assert len(a) == 138 and len(b) == 138
    assert a[0] == 0.0 and b[0] == 0.0 and b[-1] == 1.0
    assert np.all(np.diff(a[:60]) > 0)


@pytest.mark.parametrize("klev", [138, 300, 1000])
def test_finer_grids_interpolate_l137(klev):
    """The finer test grids keep the L137 model top and surface, increase
    strictly, and pass through every L137 half level whose index i * 137 /
    KLEV is whole."""
    a137, b137 = inputs.l137_ab()
    a, b = inputs.hybrid_ab(klev)
    assert len(a) == len(b) == klev + 1
    assert a[0] == a137[0] and b[0] == b137[0] and a[-1] == a137[-1] and b[-1] == b137[-1]
    assert np.all(np.diff(a + b * 101325.0) > 0)
    assert np.all(np.diff(a + b * 50000.0) > 0)
    for i in range(klev + 1):
        if (i * 137) % klev == 0:
            assert a[i] == a137[i * 137 // klev] and b[i] == b137[i * 137 // klev]
    nc = inputs.ncldtop_for(klev)
    assert 2 <= nc <= klev
    with pytest.raises(ValueError):
        inputs.hybrid_ab(1001)


@pytest.mark.parametrize("klev", [2, 60, 91, 136, 137])
def test_coarser_grids_are_subsets_of_l137(klev):
    """The coarser test grids keep the L137 model top and surface and take
    strictly increasing half levels of it."""
    a137, b137 = inputs.l137_ab()
    a, b = inputs.hybrid_ab(klev)
    assert len(a) == len(b) == klev + 1
    assert a[0] == a137[0] and b[-1] == b137[-1] and a[-1] == a137[-1]
    ph = a + b * 101325.0
    assert np.all(np.diff(ph) > 0)
    assert set(zip(a, b)) <= set(zip(a137, b137))
    nc = inputs.ncldtop_for(klev)
    assert 2 <= nc <= klev
