"""The package logger (the reference's LarmorLogger, src/larmor/_log.py)."""

import logging

LarmorLogger = logging.getLogger("larmor_b200")
LarmorLogger.addHandler(logging.NullHandler())
