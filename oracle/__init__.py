"""Oracle for the density-and-potential stage (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may use
this package, to check results or as the timed CPU baseline.  The product path
(galaxyfinder_b200 / libgf.so) never imports it.
"""
