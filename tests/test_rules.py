"""Rule strings (guiSystem.cpp:92-163), pinned by the reference's only exact-value test,
`--test cli-rules` (testRunner.cpp:231-260): "3,5-7" and "2,4" round-trip, maxCS 8 decodes; the
parser's edge forms; and, on hypothesis-drawn masks, the formatter against a restatement of
BitmaskToRuleString and the parse of its output back to the mask."""
import pytest
from hypothesis import given, settings
from hypothesis import strategies as st

import cave_b200 as cb


def test_cli_rules_known_answer():
    birth = cb.rule_string_to_bitmask("3,5-7")
    survival = cb.rule_string_to_bitmask("2,4")
    assert birth == 0b1110100 and survival == 0b1010
    assert cb.bitmask_to_rule_string(birth) == "3,5-7"
    assert cb.bitmask_to_rule_string(survival) == "2,4"
    p = cb.make_params(8, 7, birth, survival)
    assert ((p.birthAndMaxCellStateRules >> 60) & 0xF) + 1 == 8  # simulation.h:58-59


@pytest.mark.parametrize("text,mask,back", [
    ("", 0, "-"),
    ("1", 1, "1"),
    ("1,2", 0b11, "1,2"),          # a run of two is not collapsed
    ("1-3", 0b111, "1-3"),
    (" 4 , 6-8 ,10", 0b1011101000, "4,6-8,10"),
    ("0,61,5", 0b10000, "5"),      # out-of-range values are ignored
    ("5-3", 0, "-"),
    ("58-62", (1 << 57) | (1 << 58) | (1 << 59), "58-60"),
])
def test_rule_string_forms(text, mask, back):
    assert cb.rule_string_to_bitmask(text) == mask
    assert cb.bitmask_to_rule_string(mask) == back


def _format(mask):
    """guiSystem.cpp:92-123 restated: 1-based set bits below 60, runs of three or more as a-b."""
    bits = [b + 1 for b in range(60) if (mask >> b) & 1]
    if not bits:
        return "-"
    parts, i = [], 0
    while i < len(bits):
        j = i
        while j + 1 < len(bits) and bits[j + 1] == bits[j] + 1:
            j += 1
        parts += [f"{bits[i]}-{bits[j]}"] if j - i >= 2 else [str(b) for b in bits[i:j + 1]]
        i = j + 1
    return ",".join(parts)



@settings(max_examples=500, deadline=None)
@given(mask=st.one_of(st.integers(0, (1 << 64) - 1), st.integers(0, (1 << 27) - 1),
                      st.lists(st.integers(0, 59), max_size=8).map(lambda v: sum(1 << b for b in set(v)))))
def test_rule_string_round_trip(mask):
    text = cb.bitmask_to_rule_string(mask)
    assert text == _format(mask)
    assert cb.rule_string_to_bitmask(text) == (mask & ((1 << 60) - 1) if text != "-" else 0)
