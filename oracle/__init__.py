"""CPU oracle for the QVM repulsion path. TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm may
import this package, and only as the checker or the timed CPU baseline. The product
(zxtalori_b200) never imports, links or executes anything here.
"""
