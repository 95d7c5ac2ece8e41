# DMRJtensorB200.jl -- Julia host binding of libdmrgb200.so (C ABI in include/dmrg_b200.h).
#
# A drop-in for DMRJtensor's two-site ground-state path:
#   dmrg(psi::MPS, mpo::MPO; m, minm, sweeps, cutoff, silent, SvNbond)   algs/DMRG.jl:549-588
#   makeEnv(psi, mpo) / Lupdate / Rupdate                               lib/Env/makeEnv.jl:196-246
# `dmrg_b200(psi, mpo; ...)` takes the reference's own MPS/MPO objects (fields `psi.A`, `psi.oc`,
# `mpo.H`, lib/types.jl:84-101), runs every sweep on the GPU and writes the optimised tensors back
# into `psi` (dense `tens` or, for quantum-number MPS, rebuilt with `makeqMPS`), returning the
# energy exactly as `dmrg` does. Tensors cross the boundary in their dense-equivalent column-major
# form ([ml,d,mr] sites, [wl,d,d,wr] MPO sites); quantum numbers cross as integer charges
# (`charges[i]` = d x nsym Int32 matrix of site i's physical charges, the same labels that were
# given to makeqMPS / makeqMPO, e.g. 2Sz for U1 spin). All sizes are checked by the library.
module DMRJtensorB200

export dmrg_b200, B200Env, makeEnv_b200, Lupdate_b200!, Rupdate_b200!, expect_b200,
       correlationmatrix_b200, save_b200, load_b200

const libdmrg = get(ENV, "DMRG_B200_LIB", joinpath(@__DIR__, "..", "libdmrgb200.so"))

# mirrors struct dmrg_params (C layout: ints and doubles in declaration order)
mutable struct Params
  maxm::Cint
  minm::Cint
  cutoff::Cdouble
  krylov::Cint
  precision::Cint
  svnbond::Cint
  degen_rtol::Cdouble
  betatest::Cdouble
  fp64_final::Cint
  profile::Cint
  reserved::NTuple{6,Cint}
end
Params() = Params(0, 0, 0.0, 0, 0, 0, 0.0, 0.0, 0, 0, ntuple(_ -> Cint(0), 6))

# mirrors struct dmrg_sweep_stats
mutable struct SweepStats
  energy::Cdouble
  max_truncerr::Cdouble
  biggest_m::Cint
  n_matvec::Cint
  entropy::Cdouble
  seconds::Cdouble
  heff_flops::Cdouble
  heff_seconds::Cdouble
  env_flops::Cdouble
  env_seconds::Cdouble
  eig_seconds::Cdouble
  vec_seconds::Cdouble
  d_top::NTuple{8,Cdouble}
  gemm_flops::Cdouble
  gemm_seconds::Cdouble
  gemm_launches::Cint
  eig_max_n::Cint
  host_seconds::Cdouble
  wait_seconds::Cdouble
end
SweepStats() = SweepStats(0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, ntuple(_ -> 0.0, 8), 0, 0, 0, 0, 0, 0)

lasterror(ctx) = unsafe_string(ccall((:dmrg_last_error, libdmrg), Cstring, (Ptr{Cvoid},), ctx))

function check(code, ctx, what)
  code == 0 || error("libdmrgb200 $what failed (status $code): $(lasterror(ctx))")
  nothing
end

mutable struct Context
  h::Ptr{Cvoid}
end
function Context(device::Integer=0; hbm_budget_bytes::Integer=0)
  out = Ref{Ptr{Cvoid}}(C_NULL)
  code = ccall((:dmrg_ctx_create, libdmrg), Cint, (Cint, Csize_t, Ref{Ptr{Cvoid}}),
               device, hbm_budget_bytes, out)
  code == 0 || error("dmrg_ctx_create failed (status $code)")
  c = Context(out[])
  finalizer(x -> x.h == C_NULL || ccall((:dmrg_ctx_destroy, libdmrg), Cint, (Ptr{Cvoid},), x.h), c)
  c
end

# The reference stores tensors as `tens` (dense) or `Qtens`; `makeArray` (TensorPACK) gives the
# dense-equivalent Array of either. `densify` is a hook so that other containers can be passed.
densify(T) = Array{Float64}(Main.makeArray(T))

function upload_mpo(ctx::Context, mpo, charges)
  L = length(mpo.H)
  Ws = [densify(mpo.H[i]) for i = 1:L]
  d = Cint[size(W, 2) for W in Ws]
  wl = Cint[size(W, 1) for W in Ws]
  wr = Cint[size(W, 4) for W in Ws]
  nsym = charges === nothing ? 0 : size(charges[1], 2)
  ptrs = [pointer(W) for W in Ws]
  # physical charges, state-major (d*nsym ints per site); kept alive across the call
  qkeep = charges === nothing ? Matrix{Int32}[] :
          [Matrix{Int32}(permutedims(Int32.(charges[i]), (2, 1))) for i = 1:L]
  qn = charges === nothing ? Ptr{Cint}[C_NULL for _ = 1:L] : [pointer(q) for q in qkeep]
  out = Ref{Ptr{Cvoid}}(C_NULL)
  GC.@preserve Ws qkeep begin
    code = ccall((:dmrg_mpo_upload, libdmrg), Cint,
                 (Ptr{Cvoid}, Cint, Cint, Ptr{Cint}, Ptr{Cint}, Ptr{Cint}, Ptr{Ptr{Cdouble}},
                  Ptr{Ptr{Cint}}, Ptr{Ptr{Cint}}, Ref{Ptr{Cvoid}}),
                 ctx.h, L, nsym, d, wl, wr, ptrs, qn, C_NULL, out)
  end
  check(code, ctx.h, "dmrg_mpo_upload")
  out[]
end

function upload_mps(ctx::Context, hmpo, psi)
  L = length(psi.A)
  As = [densify(psi.A[i]) for i = 1:L]
  ml = Cint[size(A, 1) for A in As]
  mr = Cint[size(A, 3) for A in As]
  out = Ref{Ptr{Cvoid}}(C_NULL)
  GC.@preserve As begin
    code = ccall((:dmrg_mps_upload, libdmrg), Cint,
                 (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cint}, Ptr{Cint}, Ptr{Ptr{Cdouble}}, Ptr{Ptr{Cint}},
                  Cint, Ref{Ptr{Cvoid}}),
                 ctx.h, hmpo, ml, mr, [pointer(A) for A in As], C_NULL, psi.oc - 1, out)
  end
  check(code, ctx.h, "dmrg_mps_upload")
  out[]
end

"""
    dmrg_b200(psi, mpo; m, minm=2, sweeps=1, cutoff=0.0, silent=false, SvNbond=0, krylov=2,
              charges=nothing, Qlabels=nothing, precision=0, device=0)

Two-site DMRG of the reference's `dmrg(psi, mpo; method="twosite")` on the GPU. `charges`:
per-site d x nsym integer charges (required for quantum-number MPS; `Qlabels` are forwarded to
`makeqMPS` when the result is written back). Returns the energy of the last bond step, like `dmrg`.
"""
function dmrg_b200(psi, mpo; m::Integer=0, minm::Integer=2, sweeps::Integer=1, cutoff::Float64=0.0,
                   silent::Bool=false, SvNbond::Integer=0, krylov::Integer=2, charges=nothing,
                   Qlabels=nothing, precision::Integer=0, device::Integer=0)
  ctx = Context(device)
  hmpo = upload_mpo(ctx, mpo, charges)
  st = upload_mps(ctx, hmpo, psi)
  try
    check(ccall((:dmrg_env_build, libdmrg), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), st, hmpo), ctx.h,
          "dmrg_env_build")
    p = Params()
    ccall((:dmrg_params_default, libdmrg), Cvoid, (Ref{Params},), p)
    p.maxm, p.minm, p.cutoff, p.krylov, p.precision, p.svnbond = m, minm, cutoff, krylov, precision, SvNbond
    energy = 0.0
    for s = 1:sweeps
      stats = SweepStats()
      check(ccall((:dmrg_sweep, libdmrg), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Ref{Params}, Ref{SweepStats}),
                  st, hmpo, p, stats), ctx.h, "dmrg_sweep")
      energy = stats.energy
      silent || println("sweep $s, energy $(stats.energy), largest truncation $(stats.max_truncerr), ",
                        "m $(stats.biggest_m), entropy $(stats.entropy), $(stats.seconds) s")
    end
    write_back!(ctx, st, psi, Qlabels)
    return energy
  finally
    ccall((:dmrg_state_destroy, libdmrg), Cint, (Ptr{Cvoid},), st)
    ccall((:dmrg_mpo_destroy, libdmrg), Cint, (Ptr{Cvoid},), hmpo)
  end
end

# Downloads every site in its dense-equivalent form (bond bases grouped by charge: a gauge change
# of the same state) and stores it in psi; quantum-number states are rebuilt with makeqMPS.
function write_back!(ctx::Context, st, psi, Qlabels)
  L = length(psi.A)
  arrays = Vector{Array{Float64,3}}(undef, L)
  for i = 1:L
    ml, mr = Ref{Cint}(0), Ref{Cint}(0)
    check(ccall((:dmrg_mps_download, libdmrg), Cint,
                (Ptr{Cvoid}, Cint, Ptr{Cdouble}, Ref{Cint}, Ref{Cint}), st, i - 1, C_NULL, ml, mr),
          ctx.h, "dmrg_mps_download (sizes)")
    d = size(psi.A[i], 2)
    A = Array{Float64}(undef, ml[], d, mr[])
    check(ccall((:dmrg_mps_download, libdmrg), Cint,
                (Ptr{Cvoid}, Cint, Ptr{Cdouble}, Ref{Cint}, Ref{Cint}), st, i - 1, A, ml, mr),
          ctx.h, "dmrg_mps_download")
    arrays[i] = A
  end
  oc = Ref{Cint}(0)
  check(ccall((:dmrg_state_oc, libdmrg), Cint, (Ptr{Cvoid}, Ref{Cint}), st, oc), ctx.h, "dmrg_state_oc")
  if Qlabels === nothing
    for i = 1:L
      psi.A[i] = Main.tens(arrays[i])
    end
  else
    qpsi = Main.makeqMPS(Qlabels, Main.MPS(arrays; oc=oc[] + 1); newnorm=false)
    for i = 1:L
      psi.A[i] = qpsi.A[i]
    end
  end
  psi.oc = oc[] + 1
  psi
end

"""
    B200Env

Resident environments of one (psi, mpo) pair on the GPU: `makeEnv_b200` builds them
(makeEnv, lib/Env/makeEnv.jl:196-221), `Lupdate_b200!(i, env)` / `Rupdate_b200!(i, env)` are
Lupdate!/Rupdate! (lib/MPO_MPS/Lupdate.jl:17-37, Rupdate.jl:17-37) and `env[i, :left]` /
`env[i, :right]` download Lenv[i] / Renv[i] as dense [m, w, m] arrays.
"""
mutable struct B200Env
  ctx::Context
  mpo::Ptr{Cvoid}
  st::Ptr{Cvoid}
end

function makeEnv_b200(psi, mpo; charges=nothing, device::Integer=0)
  ctx = Context(device)
  hmpo = upload_mpo(ctx, mpo, charges)
  st = upload_mps(ctx, hmpo, psi)
  check(ccall((:dmrg_env_build, libdmrg), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), st, hmpo), ctx.h, "dmrg_env_build")
  e = B200Env(ctx, hmpo, st)
  finalizer(e) do x
    ccall((:dmrg_state_destroy, libdmrg), Cint, (Ptr{Cvoid},), x.st)
    ccall((:dmrg_mpo_destroy, libdmrg), Cint, (Ptr{Cvoid},), x.mpo)
  end
  e
end

Lupdate_b200!(i::Integer, e::B200Env) =
  check(ccall((:dmrg_lupdate, libdmrg), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Cint), e.st, e.mpo, i - 1),
        e.ctx.h, "dmrg_lupdate")
Rupdate_b200!(i::Integer, e::B200Env) =
  check(ccall((:dmrg_rupdate, libdmrg), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Cint), e.st, e.mpo, i - 1),
        e.ctx.h, "dmrg_rupdate")

function Base.getindex(e::B200Env, i::Integer, side::Symbol)
  left = side === :left ? 1 : 0
  dims = zeros(Cint, 3)
  check(ccall((:dmrg_env_get, libdmrg), Cint, (Ptr{Cvoid}, Cint, Cint, Ptr{Cdouble}, Ptr{Cint}),
              e.st, i - 1, left, C_NULL, dims), e.ctx.h, "dmrg_env_get (sizes)")
  out = Array{Float64}(undef, dims...)
  check(ccall((:dmrg_env_get, libdmrg), Cint, (Ptr{Cvoid}, Cint, Cint, Ptr{Cdouble}, Ptr{Cint}),
              e.st, i - 1, left, out, dims), e.ctx.h, "dmrg_env_get")
  out
end

# expect(psi, H) (lib/MPO_MPS/expect.jl:47-56) on the state of a B200Env: <psi|H|psi>, not
# normalised; `H` is another uploaded MPO over the same sites (default: the Env's own).
function expect_b200(e::B200Env, hmpo::Ptr{Cvoid}=e.mpo)
  v = Ref{Cdouble}(0.0)
  check(ccall((:dmrg_expect, libdmrg), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Ref{Cdouble}), e.st, hmpo, v),
        e.ctx.h, "dmrg_expect")
  v[]
end

# correlationmatrix(psi, Cc, Ca; trail) (lib/MPO_MPS/correlationmatrix.jl:21-83), operators
# O[bra, ket] as d x d Float64 matrices; the centre of the state is not moved.
function correlationmatrix_b200(e::B200Env, Cc::Matrix{Float64}, Ca::Matrix{Float64};
                                trail=nothing, L::Integer)
  d = size(Cc, 1)
  rho = Matrix{Float64}(undef, L, L)
  F = trail === nothing ? C_NULL : Matrix{Float64}(trail)
  check(ccall((:dmrg_correlationmatrix, libdmrg), Cint,
              (Ptr{Cvoid}, Cint, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}),
              e.st, d, Cc, Ca, F, rho), e.ctx.h, "dmrg_correlationmatrix")
  rho
end

# Checkpoint of the Env's device state (the persistence of largeMPS / loadMPS,
# lib/MPS/largeMPS.jl:19-81); load_b200 returns a new B200Env with rebuilt environments.
save_b200(e::B200Env, path::AbstractString) =
  check(ccall((:dmrg_state_save, libdmrg), Cint, (Ptr{Cvoid}, Cstring), e.st, path),
        e.ctx.h, "dmrg_state_save")

function load_b200(e::B200Env, path::AbstractString)
  out = Ref{Ptr{Cvoid}}(C_NULL)
  check(ccall((:dmrg_state_load, libdmrg), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Cstring, Ref{Ptr{Cvoid}}),
              e.ctx.h, e.mpo, path, out), e.ctx.h, "dmrg_state_load")
  check(ccall((:dmrg_env_build, libdmrg), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), out[], e.mpo), e.ctx.h,
        "dmrg_env_build")
  B200Env(e.ctx, e.mpo, out[])   # shares the MPO handle: no finalizer of its own
end

end # module
