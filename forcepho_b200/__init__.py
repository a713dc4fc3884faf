"""forcepho's likelihood hot path on B200 (sm_100a CUDA behind a C ABI).

Modules, with the reference counterparts they stand in for:

* ``proposal``    -- ``B200Proposer`` / ``PlainProposer`` (``forcepho.proposal.GPUProposer``)
* ``device``      -- ``B200PatchMixin`` (``forcepho.patches.device_patch.GPUPatchMixin``) and
                     ``Plan``, the device-resident work plan of many patches
* ``batch``       -- ``BatchedProposer``: one proposal for each of many patches per launch
* ``model``       -- ``FastPosterior``, ``BoundedTransform``, ``stack_grad`` (``forcepho.model``)
* ``hmc``         -- ``DeviceHMC``: HMC of many patches with all state on the device
* ``nuts``        -- ``BatchedNUTS``, ``run_nuts`` (``forcepho.fitting.run_lmc``)
* ``render``      -- ``subtract_fixed``, ``design_matrix``, ``render`` (``device_patch.py``)
* ``fitting``     -- ``optimize_one_band``, ``optimize_fluxes`` (``forcepho.fitting``)
* ``autograd``    -- ``BatchChi2`` / ``PatchChi2``: per-band chi2 of many / one patch as a
                     device-resident ``torch.autograd.Function`` of the scene parameters
* ``stores``      -- ``FITSPatch``, ``StorePatch``, ``PSFStore``, regions, and the FITS, TAN-WCS
                     and HDF5 readers (``forcepho.patches.pixel_patch``, ``storage``, ``forcepho.region``)
* ``distributed`` -- ``PatchFarm``: patches shared out over processes / GPUs
* ``superscene``  -- ``SuperScene`` / ``LinkedSuperScene``: the field's catalog, regions checked
                     out of and into it, prior bounds (``forcepho.superscene``)
* ``dispatcher``  -- rounds of checked-out regions worked as batches on every GPU
                     (``forcepho.dispatcher``)
* ``sources``, ``patch``, ``structs``, ``kernel_limits``, ``splines`` -- the data
  model (``forcepho.sources``, ``forcepho.patches.patch``, ``forcepho.kernel_limits``)
* ``synthetic``   -- seeded synthetic patches of the benchmark workloads
* ``build``, ``_native`` -- the in-tree CUDA library and its ctypes bindings
* ``phase_split`` -- the tile kernel's phase split, from the diagnostic build

Submodules are imported on use; importing the package itself loads nothing.
"""
