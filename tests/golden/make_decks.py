"""Reference outputs of the deck fixtures in tests/golden/decks/.

Runs every *.nec deck of that folder through the reference's own deck front
end (nec2++ built from the reference sources by `make -C oracle ref` into
oracle/_ref/nec2cpp) and stores its text output beside the deck as *.out.
The decks themselves are written for this repository.

    make -C oracle ref && python tests/golden/make_decks.py
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
NEC2CPP = os.path.join(ROOT, "oracle", "_ref", "nec2cpp")


def main():
    if not os.path.exists(NEC2CPP):
        sys.exit("build the reference first: make -C oracle ref")
    for deck in sorted(glob.glob(os.path.join(HERE, "decks", "*.nec"))):
        out = deck[:-4] + ".out"
        r = subprocess.run([NEC2CPP, "-i", deck, "-o", out], capture_output=True, text=True, timeout=600)
        print(f"{os.path.basename(deck):28s} rc={r.returncode} -> {os.path.basename(out)}")


if __name__ == "__main__":
    main()
