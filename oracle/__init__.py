"""CPU oracle of rsr's evaluator: TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use this
package, as the checker (and as the timed CPU baseline); the engine never does.
"""
