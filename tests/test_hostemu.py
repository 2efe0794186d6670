"""The GPU kernels' column code, compiled for the host (tests/hostemu), against
the oracle: bit-for-bit with either libm, on the metric's configuration 1 and
on the edge cases.  This proves the kernel's restatement of the reference's
logic (single fused pass over the levels, sparse 5x5 matrices, operation
order) without a GPU; the GPU tests then show the device build matches the
host build."""
import numpy as np
import pytest

from openifs_b200 import inputs
from tests import util


@pytest.fixture(scope="module")
def pp(built):
    return util.params()


@pytest.mark.parametrize("libm", ["plibm", "glibc"])
def test_config1_bit_exact(pp, libm):
    p, po = pp
    arrs = inputs.generate(100, 32, p, seed=1)
    ref, nw = util.run_oracle(po, arrs, 32, 100, 3200, libm=libm)
    emu, nwe = util.run_hostemu(p, arrs, 32, 100, 3200, libm=libm)
    for n in util.COMPARED:
        assert np.array_equal(util.defined(n, emu[n]), util.defined(n, ref[n])), n
    assert nw == nwe


@pytest.mark.parametrize("case", util.EDGE_CASES)
def test_edge_cases_bit_exact(pp, case):
    p, po = pp
    arrs = util.apply_case(inputs.generate(4, 37, p, seed=5), case)
    ngptot = 4 * 37 - 6
    ref, _ = util.run_oracle(po, arrs, 37, 4, ngptot)
    emu, _ = util.run_hostemu(p, arrs, 37, 4, ngptot)
    for n in util.COMPARED:
        assert np.array_equal(util.defined(n, emu[n]), util.defined(n, ref[n])), (case, n)


@pytest.mark.parametrize("klev", [60, 91])
def test_other_vertical_grids_bit_exact(klev):
    """Other vertical resolutions (60 and 91 levels, NCLDTOP from their own
    standard atmosphere): the kernel's column code against the oracle, bit for
    bit, with a ragged last block."""
    p, po = util.params(inputs.ncldtop_for(klev))
    arrs = inputs.generate(6, 33, p, klev=klev, seed=23)
    ngptot = 6 * 33 - 4
    ref, nw = util.run_oracle(po, arrs, 33, 6, ngptot, klev=klev)
    emu, nwe = util.run_hostemu(p, arrs, 33, 6, ngptot, klev=klev)
    for n in util.COMPARED:
        a = util.defined(n, util._valid_cols(emu[n], ngptot, 33))
        b = util.defined(n, util._valid_cols(ref[n], ngptot, 33))
        assert np.array_equal(a, b), (klev, n)
    assert nw == nwe
    assert np.abs(ref["tendency_loc_t"]).max() > 0


@pytest.mark.parametrize("case", ["clear", "supersaturated", "tiny_cloud_fraction", "negative_condensate"])
def test_optional_forms_edge_cases(pp, case):
    """The budget, SPP and inhomogeneity form on edge-case columns, with the
    kernels' fast pass and rerun: outputs, PFSD and PEXTRA bit for bit with
    the oracle."""
    p0, po0 = pp
    p, po = util.opt_params(p0, "all+budgets"), util.opt_params(po0, "all+budgets")
    arrs = util.apply_case(inputs.generate(3, 32, p, seed=47), case)
    ngptot = 3 * 32 - 2
    diag = inputs.generate_diag(arrs, 32, util.fields.budget_fields_needed(p) + 1, seed=47)
    ref, dref, nw = util.run_oracle_diag(po, arrs, diag, 32, 3, ngptot)
    emu, demu, nwe = util.run_hostemu_diag(p, arrs, diag, 32, 3, ngptot, flags=0x300)
    assert nw == nwe
    for n in util.COMPARED:
        assert np.array_equal(util.defined(n, emu[n]), util.defined(n, ref[n])), n
    assert np.array_equal(demu["pextra"], dref["pextra"])
    assert np.array_equal(demu["pfsd"], dref["pfsd"])


def test_more_levels_than_the_fast_pass_keeps():
    """300 levels, above the 256 whose PLUDE inputs the kernels' fast pass
    keeps: the kernels then run their plain column code.  The host build of
    that path (the fast-pass flag is ignored there, as on the GPU) against
    the oracle, bit for bit, in the plain FP64 form and with every budget
    section, SPP and the inhomogeneity paths on."""
    klev = 300
    p, po = util.params(inputs.ncldtop_for(klev))
    arrs = inputs.generate(3, 32, p, klev=klev, seed=31)
    ngptot = 3 * 32 - 5
    ref, nw = util.run_oracle(po, arrs, 32, 3, ngptot, klev=klev)
    emu, nwe = util.run_hostemu(p, arrs, 32, 3, ngptot, klev=klev, precision=0x300)
    for n in util.COMPARED:
        a = util.defined(n, util._valid_cols(emu[n], ngptot, 32))
        b = util.defined(n, util._valid_cols(ref[n], ngptot, 32))
        assert np.array_equal(a, b), n
    assert nw == nwe
    q, qo = util.opt_params(p, "all+budgets"), util.opt_params(po, "all+budgets")
    diag = inputs.generate_diag(arrs, 32, util.fields.budget_fields_needed(q) + 1, klev=klev, seed=31)
    ref, dref, nw = util.run_oracle_diag(qo, arrs, diag, 32, 3, ngptot, klev=klev)
    emu, demu, nwe = util.run_hostemu_diag(q, arrs, diag, 32, 3, ngptot, flags=0x300, klev=klev)
    for n in util.COMPARED:
        assert np.array_equal(util.defined(n, emu[n]), util.defined(n, ref[n])), n
    assert np.array_equal(demu["pextra"], dref["pextra"])
    assert np.array_equal(demu["pfsd"], dref["pfsd"])
    assert nw == nwe


def test_libm_sensitivity_of_the_reference(pp):
    """The reference algorithm with two correct libms (glibc and plibm, within
    1 ulp of each other) -- the spread any GPU build is measured against."""
    p, po = pp
    arrs = inputs.generate(100, 32, p, seed=1)
    a, _ = util.run_oracle(po, arrs, 32, 100, 3200, libm="plibm")
    b, _ = util.run_oracle(po, arrs, 32, 100, 3200, libm="glibc")
    rep, _ = util.compare(a, b)
    assert max(rep.values()) < 1e-8
    assert max(rep.values()) > 1e-14  # the libms do differ


def test_mixed_form_on_host(pp):
    """The FP32-mixed column code (host build, glibc float libm) against the
    FP64 oracle: species, T and surface-flux tendencies within 1e-5
    (max |err| / max |ref| per field)."""
    p, po = pp
    arrs = inputs.generate(100, 32, p, seed=1)
    ref, _ = util.run_oracle(po, arrs, 32, 100, 3200)
    emu, _ = util.run_hostemu(p, arrs, 32, 100, 3200, precision=1)
    st = util.mixed_error_stats(emu, ref)
    for k in util.MIXED_BOUNDED:
        assert st[k]["normwise_max"] <= util.MIXED_TOL, (k, st[k])
    assert np.isfinite(st["tendency_loc_a"]["normwise_max"])


@pytest.mark.parametrize("libm", ["plibm", "glibc"])
def test_satadj_bit_exact(pp, libm):
    """CLOUD_SATADJ: the kernel's point code against the oracle, bit for bit,
    on 64 blocks of 32 columns with a ragged last block."""
    p, po = pp
    arrs = inputs.generate_satadj(64, 32, p, seed=11)
    ngptot = 64 * 32 - 7
    ref, nw = util.run_oracle_satadj(po, arrs, 32, 64, ngptot, libm=libm)
    emu, nwe = util.run_hostemu_satadj(p, arrs, 32, 64, ngptot, libm=libm)
    for n in util.fields.SATADJ_OUTPUTS:
        assert np.array_equal(emu[n], ref[n]), n
    assert nw == nwe
    # the padding columns of the last block are untouched
    assert np.all(emu["tendency_loc_t"][-1, :, 32 - 7:] == 0.0)


SATADJ_CASES = ["clear", "overcast", "cold", "warm", "strong_ascent", "strong_descent", "no_forcing"]


def apply_satadj_case(a, case):
    """Turn a generated CLOUD_SATADJ input into a case its branches single out."""
    if case == "clear":  # no cloud, no condensate: only clear-air condensation
        for n in ("pa", "pl", "pi", "tendency_cml_a", "tendency_cml_l", "tendency_cml_i"):
            a[n][:] = 0.0
    elif case == "overcast":  # full cloud cover: no clear-air condensation branch
        a["pa"][:] = 1.0
        a["tendency_cml_a"][:] = 0.0
    elif case == "cold":  # below homogeneous freezing: everything goes to ice
        a["pt"][:] = np.minimum(a["pt"], 225.0)
    elif case == "warm":
        a["pt"][:] = np.maximum(a["pt"], 285.0)
    elif case == "strong_ascent":  # omega beyond the dp/dt clamp: condensation
        a["pvervel"][:] = -50.0
    elif case == "strong_descent":  # evaporation
        a["pvervel"][:] = 50.0
    elif case == "no_forcing":
        for n in ("pvervel", "phrsw", "phrlw", "tendency_vdf_t", "tendency_vdf_q"):
            a[n][:] = 0.0
        a["pludeli"][:, 2:] = 0.0
    return a


@pytest.mark.parametrize("case", SATADJ_CASES)
def test_satadj_edge_cases_bit_exact(pp, case):
    p, po = pp
    arrs = apply_satadj_case(inputs.generate_satadj(4, 37, p, seed=13), case)
    ngptot = 4 * 37 - 5
    ref, nw = util.run_oracle_satadj(po, arrs, 37, 4, ngptot)
    emu, nwe = util.run_hostemu_satadj(p, arrs, 37, 4, ngptot)
    for n in util.fields.SATADJ_OUTPUTS:
        assert np.array_equal(emu[n], ref[n]), (case, n)
    assert nw == nwe


@pytest.mark.parametrize("libm", ["plibm", "glibc"])
def test_sltend_supersat_bit_exact(pp, libm):
    """SLTEND's supersaturation adjustment (the CLOUD_SUPERSATCHECK reuse
    after the cloud scheme): the kernel's point code against the oracle."""
    p, po = pp
    arrs = inputs.generate_sltend(32, 32, p, seed=19)
    ngptot = 32 * 32 - 3
    ref = util.run_oracle_sltend(po, arrs, 32, 32, ngptot, libm=libm)
    emu = util.run_hostemu_sltend(p, arrs, 32, 32, ngptot, libm=libm)
    for n in util.fields.SLTEND_OUTPUTS:
        assert np.array_equal(emu[n], ref[n]), n
    assert (ref["padjl"] != 0).any() and (ref["padji"] != 0).any()


@pytest.mark.parametrize("flags", util.BUDGET_CASES)
def test_budget_diagnostics_bit_exact(pp, flags):
    """The cloud budget diagnostics (LCLDBUDC/L/I/T, the vertical integral;
    cloudsc.F90:3832-4110): the kernel's budget form on the host against the
    oracle, PEXTRA bit for bit; the other outputs are unchanged by the
    budgets."""
    p0, po0 = pp
    p, po = util.with_flags(p0, flags), util.with_flags(po0, flags)
    nproma, nblk = 32, 6
    ngptot = nproma * nblk - 3
    arrs = inputs.generate(nblk, nproma, p, seed=29)
    kf = util.fields.budget_fields_needed(p) + 1
    diag = inputs.generate_diag(arrs, nproma, kf, seed=29)
    ref, dref, nw = util.run_oracle_diag(po, arrs, diag, nproma, nblk, ngptot)
    emu, demu, nwe = util.run_hostemu_diag(p, arrs, diag, nproma, nblk, ngptot)
    assert nw == nwe
    assert np.array_equal(demu["pextra"], dref["pextra"])
    assert (dref["pextra"] != diag["pextra"]).any()
    plain, _ = util.run_oracle(po0, arrs, nproma, nblk, ngptot, libm="plibm")
    for n in util.COMPARED:
        assert np.array_equal(util.defined(n, emu[n]), util.defined(n, ref[n])), n
        assert np.array_equal(util.defined(n, ref[n]), util.defined(n, plain[n])), n


@pytest.mark.parametrize("case", ["budgets", "spp", "all+budgets"])
def test_optional_forms_rerun_leaves_results_unchanged(pp, case):
    """The kernels' fast pass with its rerun in the budget and SPP/
    inhomogeneity forms: with no column rerunning, with every column
    rerunning (the redo build, whose divisions all report) and with three
    columns reporting in mid-column (an out-of-window pressure at levels 60,
    90 and 120), the outputs, PFSD and PEXTRA equal the plain column code's
    and the oracle's bit for bit.  PEXTRA is accumulated in place, so the
    fast pass leaves a reporting column's levels from the report on to the
    rerun: a level added twice, or not at all, would show here."""
    p0, po0 = pp
    if case == "budgets":
        p, po = util.with_flags(p0, util.BUDGET_CASES[-1]), util.with_flags(po0, util.BUDGET_CASES[-1])
    else:
        p, po = util.opt_params(p0, case), util.opt_params(po0, case)
    nproma, nblk = 32, 6
    ngptot = nproma * nblk - 3
    arrs = util.with_out_of_window_pressure(inputs.generate(nblk, nproma, p, seed=43))
    diag = inputs.generate_diag(arrs, nproma, util.fields.budget_fields_needed(p) + 1, seed=43)
    ref, dref, nw = util.run_oracle_diag(po, arrs, diag, nproma, nblk, ngptot)
    for n in util.COMPARED:
        assert np.isfinite(util.defined(n, ref[n])).all(), n
    for libm, flags in (("plibm", 0), ("plibm", 0x200), ("plibm", 0x300), ("redo", 0x300)):
        emu, demu, nwe = util.run_hostemu_diag(p, arrs, diag, nproma, nblk, ngptot, libm=libm, flags=flags)
        assert nw == nwe, (libm, flags)
        for n in util.COMPARED:
            assert np.array_equal(util.defined(n, emu[n]), util.defined(n, ref[n])), (libm, flags, n)
        assert np.array_equal(demu["pfsd"], dref["pfsd"]), (libm, flags)
        assert np.array_equal(demu["pextra"], dref["pextra"]), (libm, flags)


@pytest.mark.parametrize("case", util.OPT_CASES)
def test_spp_inhomogeneity_bit_exact(pp, case):
    """SPP perturbations, LCLOUD_INHOMOG and LRAD_CLOUD_INHOMOG (PFSD), the
    aerosol switches (PRE_ICE, PICRIT_AER, PNICE), alone and together with the
    budgets: the kernel's OPT form on the host against the oracle, every
    output and PFSD/PEXTRA bit for bit, both libms."""
    p0, po0 = pp
    p, po = util.opt_params(p0, case), util.opt_params(po0, case)
    nproma, nblk = 32, 6
    ngptot = nproma * nblk - 3
    arrs = inputs.generate(nblk, nproma, p, seed=43)
    diag = inputs.generate_diag(arrs, nproma, util.fields.budget_fields_needed(p) + 1, seed=43)
    for libm in ("plibm", "glibc"):
        ref, dref, nw = util.run_oracle_diag(po, arrs, diag, nproma, nblk, ngptot, libm=libm)
        emu, demu, nwe = util.run_hostemu_diag(p, arrs, diag, nproma, nblk, ngptot, libm=libm)
        assert nw == nwe
        for n in util.COMPARED:
            assert np.array_equal(util.defined(n, emu[n]), util.defined(n, ref[n])), (libm, n)
        assert np.array_equal(demu["pfsd"], dref["pfsd"]), libm
        assert np.array_equal(demu["pextra"], dref["pextra"]), libm
    plain, _ = util.run_oracle(po0, arrs, nproma, nblk, ngptot, libm="plibm")
    if case != "radinhomog":  # the options change the physics
        assert any(not np.array_equal(util.defined(n, ref[n]), util.defined(n, plain[n])) for n in util.COMPARED)
    if "rad" in case or case.startswith("all"):
        fsd = dref["pfsd"][:-1]  # full blocks (the last block's padding is not written)
        assert (fsd >= 0.1).all() and (fsd <= 3.575).all() and len(np.unique(fsd)) > 10


@pytest.mark.parametrize("form", [0, 1, 2])
def test_gen_column_code_identical(pp, form):
    """The GEN column code (parameter-exponent pows without their tests for
    the exponents 0.5, 1.5, 2 and 3, which the default parameters never use)
    gives the same bits as the tested code, in every form; the FP64 form also
    equals the oracle."""
    p, po = pp
    arrs = inputs.generate(100, 32, p, seed=1)
    a, nwa = util.run_hostemu(p, arrs, 32, 100, 3200, precision=form)
    b, nwb = util.run_hostemu(p, arrs, 32, 100, 3200, precision=form | 0x100)
    for n in util.COMPARED:
        assert np.array_equal(util.defined(n, a[n]), util.defined(n, b[n])), (form, n)
    assert nwa == nwb
    if form == 0:
        ref, _ = util.run_oracle(po, arrs, 32, 100, 3200)
        for n in util.COMPARED:
            assert np.array_equal(util.defined(n, b[n]), util.defined(n, ref[n])), n


@pytest.mark.parametrize("form,gen", [(0, False), (0, True), (1, True), (2, True)])
def test_column_rerun_leaves_results_unchanged(pp, form, gen):
    """The kernels' fast pass with its rerun (flag 0x200: the fast pass keeps
    each level's PLUDE input, a column it reports runs again with IEEE
    division reading PLUDE from that copy) gives the plain column code's
    bits, both when no column reruns and when every column runs twice (the
    redo build, whose divisions all report): the rerun sees the inputs as
    they were, although the fast pass has already written PLUDE in place, and
    the warning count is the rerun's alone.  The FP64 form also equals the
    oracle."""
    p, po = pp
    arrs = util.apply_case(inputs.generate(100, 32, p, seed=1), "all_convection")
    ngptot = 3193
    flags = form | (0x100 if gen else 0)
    a, nwa = util.run_hostemu(p, arrs, 32, 100, ngptot, precision=flags)
    assert np.abs(util.defined("plude", a["plude"])).max() > 0
    for libm in ("plibm", "redo"):
        b, nwb = util.run_hostemu(p, arrs, 32, 100, ngptot, precision=flags | 0x200, libm=libm)
        for n in util.COMPARED:
            x = util.defined(n, util._valid_cols(a[n], ngptot, 32))
            y = util.defined(n, util._valid_cols(b[n], ngptot, 32))
            assert np.array_equal(x, y), (form, gen, libm, n)
        assert nwa == nwb, libm
    if form == 0:
        ref, _ = util.run_oracle(po, arrs, 32, 100, ngptot)
        for n in util.COMPARED:
            x = util.defined(n, util._valid_cols(b[n], ngptot, 32))
            y = util.defined(n, util._valid_cols(ref[n], ngptot, 32))
            assert np.array_equal(x, y), n
