"""`python -m fbls_b200 search ...`: the reference's `fbls search` command."""
import sys

from .pipeline import main

sys.exit(main())
