"""python -m fvm3d --input=case.nml: run a reference case file (fvm3d.cli)."""
import sys

from .cli import run

sys.exit(run())
