"""CPU restatement of the reference's Monte Carlo docking path (test infrastructure only).

reference_root() is where the scripts and tests that read the reference's own tree find it: the
GD_REFERENCE environment variable, else the tree the pin build (oracle/refpin/Makefile) last read,
recorded in oracle/_ref/REFERENCE; None when neither holds the reference's src/ directory, so
that whatever needs the tree skips cleanly.
"""
import os

_HERE = os.path.dirname(os.path.abspath(__file__))


def reference_root():
    root = os.environ.get("GD_REFERENCE")
    if not root:
        try:
            with open(os.path.join(_HERE, "_ref", "REFERENCE")) as f:
                root = f.read().strip()
        except OSError:
            return None
    return root if root and os.path.isdir(os.path.join(root, "src")) else None
