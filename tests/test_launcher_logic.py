"""Host logic of the launcher: the 4 L runs of L lines go to the device in
consecutive groups whose memory fits the context's free budget."""
from oidt_b200.simulation_launcher import RUN_ORDER, batch_groups


def test_all_runs_in_one_group_when_they_fit():
    assert batch_groups([5] * 8, 100) == [list(range(8))]


def test_groups_are_consecutive_and_fit():
    sizes = [3, 4, 2, 6, 1, 1, 5]
    groups = batch_groups(sizes, 7)
    assert [i for g in groups for i in g] == list(range(len(sizes)))  # order kept, nothing dropped
    for g in groups:
        assert sum(sizes[i] for i in g) <= 7 or len(g) == 1


def test_oversized_run_goes_alone():
    assert batch_groups([10, 1, 1], 5) == [[0], [1, 2]]


def test_run_order_matches_reference_launcher():
    # simulation_launcher.py:26-35: (f, i), (f, r), (b, i), (b, r) for every line
    assert [(d, k) for (_, d, k) in RUN_ORDER] == [("f", "i"), ("f", "r"), ("b", "i"), ("b", "r")]
