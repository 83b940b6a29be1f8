"""Drop-in operator classes with the reference's module layout
(processing/tomo.py, tomo_large.py, propagation.py, propagation_large.py)."""
