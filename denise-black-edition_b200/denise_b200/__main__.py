"""python -m denise_b200 <par.inp> [<workflow.inp>] [device]: the reference's main program (src/denise.c)."""
import sys

from .inversion import main

sys.exit(main())
