"""CPU oracle for the two-site DMRG hot path of DMRJtensor.jl (test infrastructure).

This package is the checker, not the product. Only ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline / reference legs of ``bench.py`` may import it. The product path
(``dmrjtensor.jl_b200``) never imports, links or executes anything here.

It restates, in numpy/scipy FP64, the reference's algorithm for the path:

* ``qtensor``  -- dense and U(1)/U(1)xU(1) block-sparse tensors with the contraction,
  truncated-SVD and truncated-eigen semantics that DMRJtensor takes from TensorPACK
  (``lib/imports.jl:44-81``).
* ``models``   -- ``makeMPO`` (``lib/MPO/makeMPO.jl:59-92``), ``heisenbergMPO``/``hubbardMPO``
  (``lib/models.jl:237-273``), operator sets (``lib/models.jl:95-164``), QN assignment of MPO
  and MPS bonds (``lib/MPO/makeqMPO.jl:23-84``, ``lib/MPS/makeqMPS.jl:26-102``).
* ``dmrg``     -- ``makeEnv``/``Lupdate``/``Rupdate`` (``lib/Env/makeEnv.jl:196-221``,
  ``lib/MPO_MPS/Lupdate.jl:17-26``, ``lib/MPO_MPS/Rupdate.jl:17-26``), ``make2site`` and
  ``simplelanczos`` (``algs/DMRG.jl:48-90``), ``twostep`` (``algs/DMRG.jl:362-405``),
  ``SvNcheck!`` (``algs/DMRG.jl:172-210``) and the ``optmps`` sweep (``algs/optimizeMPS.jl:759-849``).
* ``ed``       -- exact diagonalisation of an MPO (the ``fullH`` + ``eigen`` pattern of
  ``lib/MPO/fullmpo.jl:17-57`` / ``test/MPtask_test.jl:317-334``) for known answers.

Parity pins: the energies the reference's own tests hold (``test/MPtask_test.jl:317-334``,
``test/model_test.jl:315-365``, ``test/dmrg_test.jl:82-85``, docstring of ``lib/models.jl:225-233``).
Truncation error and entanglement entropy are not checked by any reference test and the
truncation rule lives in TensorPACK (absent), so those two invariants are pinned only by the
rule written down in ``qtensor.select_kept``.
"""
