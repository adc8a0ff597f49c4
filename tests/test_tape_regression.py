"""Slot tapes of seeded trees against the committed hashes
(tests/golden/make_tape_hashes.py): the host optimizer, walk and slot
numbering must not change a tape unless the fixture is regenerated on
purpose."""
import json
import os

import pytest

from golden.make_tape_hashes import tape_hash, trees

WANT = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "tape_hashes.json")))
TREES = trees()


@pytest.mark.parametrize("name", sorted(WANT))
def test_slot_tape_unchanged(name):
    shape, order = TREES[name]
    assert tape_hash(shape, order) == WANT[name]
