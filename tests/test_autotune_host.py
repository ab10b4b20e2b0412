"""Host-side checks of the NTT plan table (no device calls): candidate plans,
validation of plans and the set / get round trip."""
import pytest

from vortexstark_b200 import VstarkError, api


@pytest.fixture(autouse=True)
def default_plans():
    yield
    for log_n in range(5, 31):
        api.set_ntt_plan(log_n)


def test_candidates_shape():
    for log_n in range(5, 31):
        cands = api.ntt_plan_candidates(log_n)
        assert cands and len(set(cands)) == len(cands)
        for lower, items, radix in cands:
            assert items in (1, 4, 8, 16)
            if log_n <= 13:
                assert (lower, radix) == (log_n, 3)
            else:
                assert radix in (3, 5)
                assert 10 <= lower <= 13 and log_n - lower <= 11 if log_n <= 24 else lower == 13
    assert len(api.ntt_plan_candidates(20)) == 4 * 4 * 2  # lower 10..13 x items x radix
    assert len(api.ntt_plan_candidates(24)) == 8


def test_set_get_round_trip_and_defaults():
    # items 0: the default (one tile per CTA in 13-layer lower passes, 8 elsewhere)
    assert api.ntt_plan(24) == (13, 0, 3)
    assert api.ntt_plan(12) == (12, 0, 3)
    for log_n in (8, 14, 20, 24, 28):
        for plan in api.ntt_plan_candidates(log_n):
            api.set_ntt_plan(log_n, *plan)
            assert api.ntt_plan(log_n) == tuple(plan)
        api.set_ntt_plan(log_n)
    assert api.ntt_plan(20) == (13, 0, 3)


@pytest.mark.parametrize("log_n,plan", [(24, (12, 8, 3)), (20, (8, 8, 3)), (12, (10, 8, 5)), (28, (12, 8, 3)),
                                        (20, (13, 65, 3)), (20, (13, 8, 4)), (32, (0, 0, 0))])
def test_invalid_plans_rejected(log_n, plan):
    with pytest.raises(VstarkError):
        api.set_ntt_plan(log_n, *plan)


def test_merkle_split_set_get_and_tuning_file(tmp_path):
    assert api.merkle_split() == 0
    for s in range(9):
        api.set_merkle_split(s)
        assert api.merkle_split() == s
    with pytest.raises(VstarkError):
        api.set_merkle_split(9)
    api.set_ntt_plan(20, 11, 4, 5)
    path = tmp_path / "tuning.json"
    api.save_tuning(path)
    api.set_merkle_split(0)
    api.set_ntt_plan(20)
    api.load_tuning(path)
    assert api.merkle_split() == 8 and api.ntt_plan(20) == (11, 4, 5)
    api.set_merkle_split(0)
