"""The task sweep plan (vshe_layout_sweep_plan, host only): the chunks that k_trsv_task streams
through its 64 KiB shared-memory stages.  The kernel relies on these invariants for its bounds,
so they are checked here on the CPU for the sweeps the bench and the tests run:
* every staged chunk fits a stage, by the stage layout's own byte count (descriptors 16 B a
  slice, columns 4 B and values 4 or 8 B a slot, row operands 8 B (forward) or 4 + 4 or 8 B
  (backward) a row, the row range rounded out to multiples of 4), and its row range stays
  inside the vectors' 8 padding entries past n;
* a chunk that does not fit is one slice, read from global memory;
* the chunks of every task cover its slices in order, one level at a time, the last chunk of
  each level flagged; over all tasks every slice of the factor is swept exactly once;
* the slice descriptors of a chunk are its slices' offsets, widths and rows;
* every solved value a chunk's rows read comes from the same task, before the level barrier."""
import numpy as np
import pytest

from vshe import devices as D
from vshe import gpu
import oracle_api as O

STAGE = 65536
VEC_PAD = 8
LEVEL_END, DIRECT = 1, 2


def _bar():
    dev, cfg = D.config2(nx=40, ny=10, n_energies=48, L=3)
    P = O.OracleProblem(dev, cfg, O.golden_coupling(3))
    A = P.matrix(3)
    return A.rp, A.ci, P.blocks(), A.v


def _diode():
    dev, cfg = D.config1()
    P = O.OracleProblem(dev, cfg, O.golden_coupling(cfg.max_expansion_order))
    A = P.matrix(3)
    return A.rp, A.ci, P.blocks(), A.v


def _band(n=1500, width=300):
    """Lower band of `width` entries plus the diagonal and one upper entry: slices of 32 rows whose
    forward part is wider than a stage."""
    rows = []
    for i in range(n):
        rows.append(np.arange(max(0, i - width), min(n, i + 2)))
    rp = np.zeros(n + 1, np.int64)
    rp[1:] = np.cumsum([len(r) for r in rows])
    ci = np.concatenate(rows).astype(np.int32)
    v = np.where(ci == np.repeat(np.arange(n), np.diff(rp)), 4.0, -1.0 / width)
    return rp, ci, None, v


CASES = {
    "bar_block_ilu1_mixed": (_bar, dict(precond="block_ilu0", ordering="multicolor", fill_level=1), True, "mixed", 2),
    "bar_block_ilu1_fp64": (_bar, dict(precond="block_ilu0", ordering="multicolor", fill_level=1), True, "fp64", 2),
    "diode_ilu0_mixed": (_diode, dict(precond="ilu0", ordering="natural"), False, "mixed", 1),
    "diode_ilu0_fp64_per_system": (_diode, dict(precond="ilu0", ordering="natural", trsv="per_system"), False, "fp64", 1),
    "band_per_system_mixed": (_band, dict(precond="ilu0", ordering="natural", trsv="per_system"), False, "mixed", 1),
    "band_per_system_fp64": (_band, dict(precond="ilu0", ordering="natural", trsv="per_system"), False, "fp64", 1),
    "bar_slab_ilut_mixed": (_bar, dict(precond="ilut", ordering="natural", ilut_entries=20, ilut_drop=1e-3), True, "mixed", 2),
}


def _stage_bytes(ns, nslot, r0, r1, lower, vb):
    return 16 * ns + (4 + vb) * nslot + (r1 - r0) * (8 if lower else 4 + vb)


@pytest.mark.parametrize("name", sorted(CASES))
def test_sweep_plan_fits_the_stages(name):
    make, kw, blocks, precision, kind = CASES[name]
    rp, ci, bl, v = make()
    kw = dict(kw, precision=precision)
    if blocks:
        kw["blocks"] = bl
    n = len(rp) - 1
    vals = v if kw["precond"] == "ilut" else None  # the ILUT pattern comes from the values
    lay = gpu.layout(rp, ci, vals, **kw)
    plan = gpu.sweep_plan(rp, ci, vals, **kw)
    assert plan["kind"] == kind
    vb = 4 if precision == "mixed" else 8
    chunks, sdesc = plan["chunks"], plan["sdesc"]
    # level of every forward slice, from its first row
    lev_of_l = np.searchsorted(lay["lvr"], lay["lrow0"][:-1], side="right") - 1
    seen = {True: np.zeros(len(lay["loff"]) - 1, np.int64), False: np.zeros(len(lay["uoff"]) - 1, np.int64)}
    n_direct = 0
    for t in plan["tasks"]:
        for lower, c0, c1 in ((True, t[1], t[2]), (False, t[3], t[4])):
            off = lay["loff"] if lower else lay["uoff"]
            rs = lay["lrow0"] if lower else lay["uslot0"]
            prev = None
            for c in range(c0, c1):
                s0, s1, flags, nslot, o0, d0, r0, r1, rot, nbytes = [int(v) for v in chunks[c]]
                assert 0 <= s0 < s1 <= len(off) - 1 and 0 <= rot < 31
                if prev is not None and not (prev[2] & LEVEL_END):
                    assert s0 == prev[1], "chunks of one level are contiguous"
                seen[lower][s0:s1] += 1
                if lower:
                    assert np.all(lev_of_l[s0:s1] == lev_of_l[s0]), "a chunk never spans two levels"
                    if prev is not None and not (prev[2] & LEVEL_END):
                        assert lev_of_l[s0] == lev_of_l[prev[0]]
                if flags & DIRECT:
                    n_direct += 1
                    assert s1 == s0 + 1
                    one = _stage_bytes(1, off[s0 + 1] - off[s0], rs[s0] & ~3, (rs[s0 + 1] + 3) & ~3, lower, vb)
                    assert one > STAGE
                else:
                    assert nslot == off[s1] - off[s0] and o0 == off[s0]
                    assert r0 == (rs[s0] & ~3) and r1 == ((rs[s1] + 3) & ~3)
                    assert 0 <= r0 <= r1 <= n + VEC_PAD
                    assert nbytes == _stage_bytes(s1 - s0, nslot, r0, r1, lower, vb) <= STAGE
                    for k, i in enumerate(range(s0, s1)):
                        soff, width, dr0, nr = [int(v) for v in sdesc[d0 + k]]
                        assert soff == off[i] - off[s0] and width * 32 == off[i + 1] - off[i]
                        assert dr0 == rs[i] and nr == rs[i + 1] - rs[i] and 1 <= nr <= 32
                prev = (s0, s1, flags)
            if c1 > c0:
                assert chunks[c1 - 1][2] & LEVEL_END, "the last chunk of a task's sweep ends a level"
    assert np.all(seen[True] == 1) and np.all(seen[False] == 1), "every slice swept exactly once"
    if name.startswith("band"):
        assert n_direct > 0


@pytest.mark.parametrize("name", ["bar_block_ilu1_mixed", "diode_ilu0_mixed", "band_per_system_fp64", "bar_slab_ilut_mixed"])
def test_sweep_plan_honours_every_dependency(name):
    """Every factor entry a chunk's row reads (a solved value of the same sweep) belongs to a row
    of the same task swept in an earlier level of that task: tasks never wait on each other, and
    a level's rows only read rows before the level barrier."""
    make, kw, blocks, precision, kind = CASES[name]
    rp, ci, bl, v = make()
    kw = dict(kw, precision=precision)
    if blocks:
        kw["blocks"] = bl
    n = len(rp) - 1
    vals = v if kw["precond"] == "ilut" else None  # the ILUT pattern comes from the values
    lay = gpu.layout(rp, ci, vals, **kw)
    plan = gpu.sweep_plan(rp, ci, vals, **kw)
    # backward slot of every solver row
    slot_of_row = np.empty(n, np.int64)
    slot_of_row[lay["urow"]] = np.arange(n)
    for lower in (True, False):
        off = lay["loff"] if lower else lay["uoff"]
        rs = lay["lrow0"] if lower else lay["uslot0"]
        col = lay["lcol"] if lower else lay["ucol"]
        nsl = len(off) - 1
        task_of = np.full(nsl, -1)
        step_of = np.full(nsl, -1)
        for ti, t in enumerate(plan["tasks"]):
            c0, c1 = (t[1], t[2]) if lower else (t[3], t[4])
            step = 0
            for c in range(c0, c1):
                s0, s1, flags = [int(v) for v in plan["chunks"][c][:3]]
                task_of[s0:s1] = ti
                step_of[s0:s1] = step
                step += 1 if flags & LEVEL_END else 0
        assert np.all(task_of >= 0)
        # the slice holding every solver row (forward) or every backward slot
        pos = np.arange(n) if lower else slot_of_row
        slice_of_pos = np.searchsorted(rs, np.arange(n), side="right") - 1
        for j in range(nsl):
            cols = col[off[j]:off[j + 1]]
            cols = cols[cols < n]
            if cols.size == 0:
                continue
            dep = slice_of_pos[pos[cols]]
            assert np.all(task_of[dep] == task_of[j]), ("cross-task read", lower, j)
            assert np.all(step_of[dep] < step_of[j]), ("read inside its own level", lower, j)
