"""`python -m shaderous_b200 run|sweep|describe ...`: the command-line runner (cli.py)."""
import sys

from .cli import main

sys.exit(main())
