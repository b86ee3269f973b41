"""CPU restatement of the reference's Monte Carlo docking path (test infrastructure only).

reference_root() is where the scripts and builds that read the reference's own tree find it:
the GD_REFERENCE environment variable, else the checkout location the recipes of this
repository were written against; None when neither holds the reference's src/ directory, so
that whatever needs the tree skips cleanly.
"""
import os

DEFAULT_REFERENCE = "/root/reference"


def reference_root():
    root = os.environ.get("GD_REFERENCE") or DEFAULT_REFERENCE
    return root if os.path.isdir(os.path.join(root, "src")) else None
