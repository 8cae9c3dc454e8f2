"""The cell loop divides the gathered neighbour sum and the field deltas by
the number of empty faces n (spatial.rs:56-110).  For n = 3, 5 and 6 it uses
a reciprocal and one exact-remainder correction instead of an IEEE division.
That replacement must give the IEEE result for every input it is used on:
the library checks every finite float against the IEEE operator."""
import pytest

pytestmark = pytest.mark.gpu


def test_small_divisor_division_is_ieee_for_every_float(marl):
    assert marl.selftest_small_division() == 0
