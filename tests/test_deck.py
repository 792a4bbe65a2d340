"""Deck-file front end (nec_run_deck / necpp_b200/nec2b200): card parsing
and job control on the CPU; on the GPU, the result sections of every deck
in tests/golden/decks against the reference's own nec2++ output of the same
deck (tests/golden/make_decks.py), compared as the reference's nec2diff
compares outputs, field by field at the printed precision."""
import ctypes as C
import glob
import os

import pytest

from deck_sections import rel_diff, sections

HERE = os.path.dirname(os.path.abspath(__file__))
DECKS = sorted(glob.glob(os.path.join(HERE, "golden", "decks", "*.nec")))


def _run(nb, tmp_path, text_or_path, name="deck"):
    if os.path.exists(str(text_or_path)):
        deck = str(text_or_path)
    else:
        deck = str(tmp_path / (name + ".nec"))
        with open(deck, "w") as f:
            f.write(text_or_path)
    out = str(tmp_path / (name + ".out"))
    nb.lib.nec_deck_error.restype = C.c_char_p
    rc = nb.lib.nec_run_deck(deck.encode(), out.encode())
    with open(out) as f:
        return rc, f.read(), nb.lib.nec_deck_error().decode()


def test_comment_cards_must_end_with_ce(nb, tmp_path):
    rc, _, err = _run(nb, tmp_path, "CM a comment\nGW 1 5 0 0 -1 0 0 1 0.001\nGE 0\nEN\n")
    assert rc == 1 and "INCORRECT LABEL FOR A COMMENT CARD" in err


def test_unknown_and_out_of_scope_cards(nb, tmp_path):
    rc, _, err = _run(nb, tmp_path, "CM x\nCE\nGW 1 5 0 0 -1 0 0 1 0.001\nGX 1 110\nGE 0\nEN\n")
    assert rc == 1 and "GX is not part of the B200" in err
    rc, _, err = _run(nb, tmp_path, "CM x\nCE\nGW 1 5 0 0 -1 0 0 1 0.001\nGE 0\nZZ 1\nEN\n")
    assert rc == 1 and "FAULTY DATA CARD LABEL" in err
    rc, _, err = _run(nb, tmp_path, "CM x\nCE\nGW 1 5.5 0 0 -1 0 0 1 0.001\nGE 0\nEN\n")
    assert rc == 1 and "INTEGER FIELD" in err
    rc, _, err = _run(nb, tmp_path, "CM x\nCE\nGW 1 5 0 0 -1 0 0 1 0.001\nGE 0\nCP 1 1 1 2\nEN\n")
    assert rc == 1 and "CP is not part of the B200" in err


def test_geometry_errors_are_reported(nb, tmp_path):
    # a tapered wire (radius 0) needs its GC card
    rc, _, err = _run(nb, tmp_path, "CM x\nCE\nGW 1 5 0 0 -1 0 0 1 0.0\nGE 0\nEN\n")
    assert rc == 1 and "GEOMETRY DATA CARD ERROR" in err
    rc, _, err = _run(nb, tmp_path, "CM x\nCE\nGA 1 5 0.3 0.0 400.0 0.001\nGE 0\nEN\n")
    assert rc == 1 and "ARC ANGLE EXCEEDS 360 DEGREES" in err


def test_free_format_fields_and_job_end_without_execution(nb, tmp_path):
    """Comma- or blank-separated fields, lower-case mnemonics; a job with no
    execution card produces no result sections."""
    rc, text, err = _run(nb, tmp_path, "CM x\nCE\ngw 1,5,0,0,-1, 0,0,1, 0.001\nGE 0\nFR 0 1 0 0 150\nEN\n")
    assert rc == 0, err
    s = sections(text)
    assert not s["inputs"] and not s["patterns"]


def _close(a, b, tol):
    return all(rel_diff(x, y) <= tol for x, y in zip(a, b)) and len(a) == len(b)


@pytest.mark.gpu
@pytest.mark.parametrize("deck", DECKS, ids=[os.path.basename(d) for d in DECKS])
def test_deck_matches_reference_output(nb, tmp_path, deck):
    rc, text, err = _run(nb, tmp_path, deck, os.path.basename(deck)[:-4])
    assert rc == 0, err
    with open(deck[:-4] + ".out") as f:
        ref = sections(f.read())
    ours = sections(text)
    for key in ("inputs", "budgets", "patterns", "near"):
        assert len(ours[key]) == len(ref[key]), key
    # antenna inputs: tag, segment, V, I, Z, Y, power at 5 significant digits
    for a, b in zip(ours["inputs"], ref["inputs"]):
        assert len(a) == len(b)
        for ra, rb in zip(a, b):
            assert ra[:2] == rb[:2]
            assert _close(ra[2:], rb[2:], 2e-4), (ra, rb)
    for a, b in zip(ours["budgets"], ref["budgets"]):
        assert _close(a[:4], b[:4], 2e-4) and abs(a[4] - b[4]) <= 0.011, (a, b)
    # patterns: angles exact, gains to the printed 0.01 dB, fields at 5 digits
    for a, b in zip(ours["patterns"], ref["patterns"]):
        assert len(a) == len(b)
        for ra, rb in zip(a, b):
            assert ra[:2] == rb[:2]
            assert all(abs(x - y) <= 0.011 for x, y in zip(ra[2:5], rb[2:5])), (ra, rb)
            assert abs(ra[5] - rb[5]) <= 2e-4, (ra, rb)
            # |E_theta|, |E_phi| (the last four numbers: mag, phase, mag, phase)
            assert rel_diff(ra[-4], rb[-4]) <= 2e-4 and rel_diff(ra[-2], rb[-2]) <= 2e-4, (ra, rb)
    for (ka, a), (kb, b) in zip(ours["near"], ref["near"]):
        assert ka == kb and len(a) == len(b)
        for ra, rb in zip(a, b):
            assert all(abs(x - y) <= 1e-4 for x, y in zip(ra[:3], rb[:3]))
            for m in (3, 5, 7):
                assert rel_diff(ra[m], rb[m]) <= 2e-4, (ra, rb)
