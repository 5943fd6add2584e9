"""Host-side logic of the device-driven loops, on CPU: the replay lengths
of forward()'s graphs and the adjoint gather's block count."""
import math

from diffswe2d_b200.adjoint import level_blocks
from diffswe2d_b200.solver import replay_length, replay_lengths


def test_replay_lengths_halve_while_even():
    assert replay_lengths(32) == [32, 16, 8, 4, 2]
    assert replay_lengths(64) == [64, 32, 16, 8, 4, 2]
    assert replay_lengths(8) == [8, 4, 2]
    assert replay_lengths(2) == [2]
    assert replay_lengths(6) == [6]  # 6 / 2 = 3 would leave the state in the other buffer
    for chunk in (2, 4, 6, 8, 12, 16, 24, 32, 48, 64):
        assert all(n % 2 == 0 for n in replay_lengths(chunk))


def test_replay_length_is_the_longest_that_fits():
    sizes = replay_lengths(32)
    assert replay_length(sizes, math.inf) == 32
    assert replay_length(sizes, 40.0) == 32
    assert replay_length(sizes, 31.9) == 16
    assert replay_length(sizes, 9.5) == 8
    assert replay_length(sizes, 4.0) == 4
    assert replay_length(sizes, 1.2) == 2  # at least the shortest graph
    assert replay_length(sizes, 0.0) == 2


def test_replay_lengths_cover_a_call_with_few_idle_steps():
    """Greedy replays for a call of n steps (the dt known exactly) run at
    most one step past its end."""
    sizes = replay_lengths(32)
    for n in range(1, 200):
        done, left = 0, float(n)
        while done < n:
            m = replay_length(sizes, left)
            done += m
            left = n - done
        assert done - n <= 1


def test_level_blocks_one_cell_per_thread_up_to_1024():
    assert level_blocks(1, 1) == 1
    assert level_blocks(16, 16) == 1
    assert level_blocks(244, 393) == math.ceil(244 * 393 / 256)
    assert level_blocks(4096, 4096) == 1024
