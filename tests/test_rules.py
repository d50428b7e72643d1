"""Rule strings (guiSystem.cpp:92-163), pinned by the reference's only exact-value test,
`--test cli-rules` (testRunner.cpp:231-260): "3,5-7" and "2,4" round-trip, maxCS 8 decodes."""
import pytest

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
