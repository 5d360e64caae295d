"""k_p1 launch shapes and the autotuner: a shape changes how a level's
candidates are cut into tiles and how many CTAs take them, never the result.
Every shape is checked bit-exact against the built-in shape (itself checked
against the oracle), the small cases against the oracle directly."""
import pytest

import oracle
import vfb_b200
from vfb_b200 import synth
from tests import cases

pytestmark = pytest.mark.gpu

BANDS = vfb_b200.TUNE_BANDS


def _uniform(rows, tiles_log2, blocks):
    return {"rows": [rows] * BANDS, "tiles_log2": [tiles_log2] * BANDS, "blocks": [blocks] * BANDS}


SHAPES = {
    "one_row_one_cta": _uniform(1, 1, 1),
    "rows4_many_tiles_3ctas": _uniform(4, 14, 3),
    "rows16_tiles256_per_sm": _uniform(16, 8, 148),
    "rows32_no_shrink": _uniform(32, 1, 0),
    # alternating bands: consecutive levels of one solve take different shapes
    "mixed": {"rows": [1 << (b % 6) for b in range(BANDS)],
              "tiles_log2": [4 + (b % 9) for b in range(BANDS)],
              "blocks": [(0, 1, 7, 64)[b % 4] for b in range(BANDS)]},
}


def _same(a, b):
    assert a.status == b.status
    assert a.size == b.size
    assert a.rpn == b.rpn
    assert a.level_rows == b.level_rows
    assert a.level_cands == b.level_cands
    assert a.solution_index == b.solution_index


def _problems():
    insts = [synth.config_small()] + cases.small_exact_cases()[1:5] + cases.planted_cases(4)
    insts.append(cases.relaxed_cases(3)[0])
    return [vfb_b200.Problem.from_instance(i) for i in insts], insts


@pytest.fixture(scope="module")
def reference_results():
    probs, insts = _problems()
    with vfb_b200.Engine() as eng:
        return [eng.solve(p) for p in probs]


@pytest.mark.parametrize("name", list(SHAPES))
def test_shape_keeps_results(reference_results, name):
    probs, _ = _problems()
    with vfb_b200.Engine() as eng:
        eng.set_tune(SHAPES[name])
        assert eng.get_tune()["rows"] == SHAPES[name]["rows"]
        for p, want in zip(probs, reference_results):
            _same(eng.solve(p), want)
        # the batched graph takes the largest CTA request of the step
        for got, want in zip(eng.batch_solve(probs), reference_results):
            _same(got, want)


def test_shape_small_cases_equal_oracle():
    with vfb_b200.Engine() as eng:
        eng.set_tune(SHAPES["mixed"])
        for inst in cases.small_exact_cases():
            got = eng.solve(vfb_b200.Problem.from_instance(inst))
            ref = oracle.solve(oracle.Problem.from_instance(inst))
            assert got.rpn == ref["rpn"]
            assert got.level_rows == ref["level_rows"]
            assert got.level_cands == ref["level_cands"]


def test_planted_config_under_shapes():
    prob = vfb_b200.Problem.from_instance(synth.config_planted())
    with vfb_b200.Engine() as eng:
        want = eng.solve(prob)
        for name in ("rows4_many_tiles_3ctas", "mixed"):
            eng.set_tune(SHAPES[name])
            _same(eng.solve(prob), want)
        eng.set_tune(None)
        assert eng.get_tune()["rows"] == [0] * BANDS


def test_tune_set_rejects_bad_shapes():
    with vfb_b200.Engine() as eng:
        with pytest.raises(vfb_b200.VfbError):
            eng.set_tune(_uniform(3, 10, 0))      # staged rows must be a power of two
        with pytest.raises(vfb_b200.VfbError):
            eng.set_tune(_uniform(64, 10, 0))     # at most 32 staged rows
        with pytest.raises(vfb_b200.VfbError):
            eng.set_tune(_uniform(8, 41, 0))      # tile target at most 2^40
        assert eng.get_tune()["rows"] == [0] * BANDS


def test_autotune(reference_results):
    probs, _ = _problems()
    sample = [probs[0], probs[5], probs[6]]
    with vfb_b200.Engine() as eng:
        table = eng.autotune(sample, reps=1)
        assert eng.get_tune()["rows"] == table["rows"]
        tuned = [b for b in range(BANDS) if table["levels"][b]]
        assert tuned, "the sample's levels fall in some band"
        for b in range(BANDS):
            assert table["rows"][b] in (0, 2, 4, 8, 16)
            assert table["tiles_log2"][b] in (0, 8, 10, 12, 14)
            if table["levels"][b]:
                # the chosen shape is the fastest measured, the built-in one among them
                assert 0 < table["ms"][b] <= table["ms_default"][b]
            else:
                assert table["rows"][b] == 0 and table["ms"][b] == 0
        # solves and batches under the tuned table still equal the reference
        for p, want in zip(probs, reference_results):
            _same(eng.solve(p), want)
        for got, want in zip(eng.batch_solve(probs), reference_results):
            _same(got, want)
        # the profile of the context is left as it was (not enabled)
        assert eng.profile() == []
