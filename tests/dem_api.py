"""Import of the product package (its directory name is not an identifier)."""
from __future__ import annotations

import importlib
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

dem = importlib.import_module("dem-rock-calibration_b200")
