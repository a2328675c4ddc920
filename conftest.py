# Puts the in-tree package directory on sys.path for tests and tools run
# from the repository root.
import sys
from pathlib import Path

_PKG = Path(__file__).resolve().parent / "mojo-align_b200"
if str(_PKG) not in sys.path:
    sys.path.insert(0, str(_PKG))
