"""Builds the cuFFT reference harness: ``python -m cufft_ref.build`` from tests/."""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

if __name__ == "__main__":
    import cufft_ref
    print(cufft_ref.build())
