"""``python -m mcmtop_b200 i=<deck> [o=<out>] [precision=fp64|fast|mixed] [dir=<dir>] [steps=<n>]``."""
import sys

from .run import main

sys.exit(main())
