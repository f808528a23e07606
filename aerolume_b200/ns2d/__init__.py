"""The 2D step (Aerolume ns2d/core.py step_full) on sm_100a behind the C ABI."""
