"""ORACLE — test infrastructure only.

CPU restatement of FerriX's linear-static / NLGEOM *STATIC path (parser,
C3D4/C3D20 element routines, serial assembly, penalty BCs, Newton driver)
with an FP64 multifrontal sparse Cholesky in place of faer's sp_cholesky.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
import it, and only as the checker or the timed CPU baseline; the product
package ferrix_b200 never imports it.
"""
