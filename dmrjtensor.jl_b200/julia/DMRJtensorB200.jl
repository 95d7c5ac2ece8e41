# DMRJtensorB200.jl -- Julia host binding of libdmrgb200.so (C ABI in include/dmrg_b200.h).
#
# A drop-in for DMRJtensor's ground-state and TDVP paths. Loading this module after DMRJtensor adds
#   * a method of DMRJtensor.dmrg for the concrete MPS/MPO types (algs/DMRG.jl:549-588): the same
#     call, dmrg(psi, mpo; m (or maxm), minm, sweeps, cutoff, silent, goal, cvgE, SvNbond, method,
#     noise, noise_goal, noise_incr), runs every sweep of method "twosite" or "3S" on the GPU,
#     writes the optimised tensors back into psi and sets psi.oc as optmps leaves it; other methods
#     go to the reference's own implementation (`invoke` on the abstract signature), so no call
#     site changes;
#   * methods of DMRJtensor.tdvp_twosite and DMRJtensor.tdvp (algs/time.jl:211-363) that run on
#     the GPU for a real prefactor (imaginary-time evolution) and real tensors; a complex
#     prefactor or complex tensors go to the reference's implementation;
#   * the Env API on device-resident environments (lib/Env/makeEnv.jl:196-246,
#     lib/MPO_MPS/Lupdate.jl:17-37, Rupdate.jl:17-37): makeEnv_b200(psi, mpo) returns (Lenv, Renv)
#     whose Lenv[i] / Renv[i] download the dense-equivalent tensor, and Lupdate!(i, Lenv, psi, mpo)
#     / Rupdate!(i, Renv, psi, mpo) methods for them; Lupdate(L, dualpsi, psi, W) /
#     Rupdate(R, dualpsi, psi, W) on dense Float64 arrays computed on the device.
# Quantum-number MPS cross the boundary in block form: the Qtens blocks (.T, .ind, .currblock,
# the fields the reference itself reads in lib/MPS/makeqMPS.jl:62-99 and lib/MPO/MPO.jl:85-92)
# are scattered straight into the library's block layout (dmrg_mps_upload_blocks), so no
# dense-equivalent site array is built on the way in. Bond charges are propagated from the left
# edge with the integer physical charges (q(right) = q(left) + p(s)), which come from the
# `charges` keyword (d x nsym integer matrix per site, or one for all sites) or, when it is not
# given, from `qnum_ints(getQnum(2, s, psi[i]))`, a hook a program overrides for its own @makeQNs
# type. The MPO (w x d x d x w per site) crosses in dense form.
module DMRJtensorB200

import DMRJtensor

export dmrg_b200, tdvp_b200, makeEnv_b200, B200Env, B200Side, expect_b200, correlationmatrix_b200,
       correlation_b200,
       save_b200, load_b200

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
  cvgE::Cint
  tune::Cint
  goal::Cdouble
  graph::Cint
  halfsweep::Cint
end
Params() = Params(0, 0, 0.0, 0, 0, 0, 0.0, 0.0, 0, 0, 0, 0, 0.0, 0, 0)

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
  converged::Cint
  graph_launches::Cint
  cvg_check::Cdouble
end
SweepStats() = SweepStats(0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, ntuple(_ -> 0.0, 8), 0, 0, 0, 0, 0, 0,
                          0, 0, 0)

# mirrors struct dmrg_noise (the 3S schedule: noise = alpha, noise_goal, noise_incr)
mutable struct Noise
  noise::Cdouble
  noise_goal::Cdouble
  noise_incr::Cdouble
  reserved::Cdouble
end
Noise() = Noise(1.0, 0.3, 0.01, 0.0)

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

const default_ctx = Ref{Union{Nothing,Context}}(nothing)
context(device::Integer) = (default_ctx[] === nothing && (default_ctx[] = Context(device));
                            default_ctx[])

# ------------------------------------------------------------------------ tensors and charges

isqtens(T) = T isa DMRJtensor.Qtens
# dense-equivalent Array of a dense tensor (tens or Array) or an MPO site
densify(T) = T isa Array ? Array{Float64}(T) : Array{Float64}(DMRJtensor.makeArray(T))

"""
    qnum_ints(q) -> Vector{Int}

Integer charges of a quantum-number label (one entry per U(1) factor). Override this for the
label type your program's `@makeQNs` defines when `charges` is not passed to `dmrg`.
"""
qnum_ints(q) = error("qnum_ints is not defined for $(typeof(q)); pass charges= to dmrg, or " *
                     "define DMRJtensorB200.qnum_ints for this label type")

# per-site d x nsym integer charges, from `charges` or from the MPS's own physical labels
function site_charges(psi, charges)
  L = length(psi.A)
  if charges !== nothing
    return charges isa AbstractMatrix ? [Matrix{Int}(charges) for _ = 1:L] :
           [Matrix{Int}(charges[(i - 1) % length(charges) + 1]) for i = 1:L]
  end
  isqtens(psi.A[1]) || return nothing
  return [begin
            d = size(psi.A[i], 2)
            rows = [qnum_ints(DMRJtensor.getQnum(2, s, psi.A[i])) for s = 1:d]
            Matrix{Int}(permutedims(hcat(rows...), (2, 1)))
          end for i = 1:L]
end

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

function upload_dense_mps(ctx::Context, hmpo, psi)
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

# Every stored entry of a Qtens site tensor A[a, s, b] as (a, s, b, value), 1-based: block q of
# A.T has rows indexed by the tensor indices A.currblock[1] and columns by A.currblock[2]; the
# 0-based positions of entry r of a group are the column A.ind[q][g][:, r].
function foreach_entry(f, A)
  cb = A.currblock
  full = zeros(Int, 3)
  for q = 1:length(A.T)
    B = A.T[q]
    rows, cols = A.ind[q][1], A.ind[q][2]
    for c = 1:size(B, 2), r = 1:size(B, 1)
      for (k, x) in enumerate(cb[1]); full[x] = rows[k, r] + 1; end
      for (k, x) in enumerate(cb[2]); full[x] = cols[k, c] + 1; end
      f(full[1], full[2], full[3], B[r, c])
    end
  end
end

struct BondSectors
  q::Vector{Vector{Int}}      # sector charges, strictly increasing (lexicographic)
  dim::Vector{Int}
  sector::Vector{Int}         # state -> sector (1-based)
  pos::Vector{Int}            # state -> position inside its sector (0-based)
end

function group_bond(labels::Vector{Vector{Int}})
  qs = sort(unique(labels))
  idx = Dict(q => k for (k, q) in enumerate(qs))
  dim = zeros(Int, length(qs))
  sector = zeros(Int, length(labels))
  pos = zeros(Int, length(labels))
  for (x, l) in enumerate(labels)            # states keep their order inside a sector
    k = idx[l]
    sector[x] = k
    pos[x] = dim[k]
    dim[k] += 1
  end
  BondSectors(qs, dim, sector, pos)
end

# Block-form upload of a Qtens MPS (dmrg_mps_upload_blocks): bond charges propagated from the
# left edge, then every stored entry scattered into the canonical block order (for each left
# sector, for each physical state s, the [dim ka x dim kb] column-major block of the right sector
# q(ka) + p(s)).
function upload_qn_mps(ctx::Context, hmpo, psi, ch)
  L = length(psi.A)
  nsym = size(ch[1], 2)
  labels = Vector{Vector{Vector{Int}}}(undef, L + 1)
  labels[1] = [zeros(Int, nsym)]
  for i = 1:L
    A = psi.A[i]
    lab = [zeros(Int, nsym) for _ = 1:size(A, 3)]   # states no block touches keep charge 0
    foreach_entry(A) do a, s, b, v
      lab[b] = labels[i][a] .+ ch[i][s, :]
    end
    labels[i + 1] = lab
  end
  bonds = [group_bond(labels[b]) for b = 1:L + 1]
  data = Vector{Vector{Float64}}(undef, L)
  for i = 1:L
    Bl, Br = bonds[i], bonds[i + 1]
    d = size(ch[i], 1)
    rq = Dict(q => k for (k, q) in enumerate(Br.q))
    off = Dict{Tuple{Int,Int},Int}()
    n = 0
    for ka = 1:length(Bl.q), s = 1:d
      kb = get(rq, Bl.q[ka] .+ ch[i][s, :], 0)
      kb == 0 && continue
      off[(ka, s)] = n
      n += Bl.dim[ka] * Br.dim[kb]
    end
    buf = zeros(Float64, n)
    foreach_entry(psi.A[i]) do a, s, b, v
      ka = Bl.sector[a]
      o = get(off, (ka, s), -1)
      o < 0 && (v == 0 || error("site $i: entry ($a,$s,$b) violates the charges"); return)
      buf[o + Bl.pos[a] + Br.pos[b] * Bl.dim[ka] + 1] = v
    end
    data[i] = buf
  end
  nsec = Cint[length(b.q) for b in bonds]
  qn = [Cint[x for q in b.q for x in q] for b in bonds]
  dims = [Cint.(b.dim) for b in bonds]
  out = Ref{Ptr{Cvoid}}(C_NULL)
  GC.@preserve qn dims data begin
    code = ccall((:dmrg_mps_upload_blocks, libdmrg), Cint,
                 (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cint}, Ptr{Ptr{Cint}}, Ptr{Ptr{Cint}},
                  Ptr{Ptr{Cdouble}}, Cint, Ref{Ptr{Cvoid}}),
                 ctx.h, hmpo, nsec, [pointer(x) for x in qn], [pointer(x) for x in dims],
                 [pointer(x) for x in data], psi.oc - 1, out)
  end
  check(code, ctx.h, "dmrg_mps_upload_blocks")
  out[]
end

upload_mps(ctx, hmpo, psi, ch) =
  (ch !== nothing && isqtens(psi.A[1])) ? upload_qn_mps(ctx, hmpo, psi, ch) :
                                          upload_dense_mps(ctx, hmpo, psi)

# ------------------------------------------------------------------------ dmrg

function run_sweeps!(ctx, st, hmpo, p::Params, sweeps, silent, nz::Union{Nothing,Noise}=nothing)
  energy = 0.0
  for s = 1:sweeps
    stats = SweepStats()
    if nz === nothing
      check(ccall((:dmrg_sweep, libdmrg), Cint,
                  (Ptr{Cvoid}, Ptr{Cvoid}, Ref{Params}, Ref{SweepStats}), st, hmpo, p, stats),
            ctx.h, "dmrg_sweep")
    else
      check(ccall((:dmrg_sweep3s, libdmrg), Cint,
                  (Ptr{Cvoid}, Ptr{Cvoid}, Ref{Params}, Ref{Noise}, Ref{SweepStats}),
                  st, hmpo, p, nz, stats), ctx.h, "dmrg_sweep3s")
    end
    energy = stats.energy
    if !silent    # dmrgcvg's report (algs/DMRG.jl:614-620)
      println("Sweep $s (back and forth): $(round(stats.seconds, digits=5)) sec")
      println("Largest truncation = $(stats.max_truncerr), m = $(stats.biggest_m)")
      println("Energy at sweep $s is $(round(stats.energy, digits=12))")
      nz === nothing || println("(alpha = $(round(nz.noise, digits=5)))")
      println()
    end
    if stats.converged != 0
      silent || println("DMRG converged to a difference of $(stats.cvg_check) after $s sweeps!\n")
      break
    end
  end
  energy
end

"""
    dmrg(psi, mpo; m, maxm, minm=2, sweeps, cutoff, silent, goal, cvgE, SvNbond, method="twosite",
         noise, noise_goal, noise_incr, krylov=2, precision=0, charges=nothing, device=0, kwargs...)

The reference's `dmrg` (algs/DMRG.jl:549-588) for `method = "twosite"` and `method = "3S"` on the
GPU; defaults come from `algvars(psi)` as in the reference. `m` and `maxm` are the same keyword.
`krylov > 2` runs Lanczos with full re-orthogonalisation instead of the reference's 2-vector step
(the 3S step always uses a Krylov space of max(2, krylov) vectors, the reference's `r`);
`precision = 1` (3xTF32) or `2` (BF16x9) selects the split-precision contractions. Other methods
run the reference's own code.
"""
function DMRJtensor.dmrg(psi::DMRJtensor.matrixproductstate, mpo::DMRJtensor.matrixproductoperator;
                         params=DMRJtensor.algvars(psi), method::String="twosite",
                         m::Integer=params.maxm, maxm::Integer=m, minm::Integer=2,
                         sweeps::Integer=params.sweeps, cutoff::Float64=params.cutoff,
                         silent::Bool=params.silent, goal::Float64=params.goal,
                         cvgE::Bool=params.cvgE, SvNbond::Integer=params.SvNbond,
                         noise::Number=first(params.noise), noise_goal::Float64=params.noise_goal,
                         noise_incr::Float64=params.noise_incr,
                         halfsweep::Bool=params.halfsweep,
                         krylov::Integer=2, precision::Integer=0, charges=nothing,
                         device::Integer=0, kwargs...)
  if method != "twosite" && method != "3S"
    return invoke(DMRJtensor.dmrg, Tuple{DMRJtensor.MPS,DMRJtensor.MPO}, psi, mpo;
                  params=params, method=method, m=maxm, minm=minm, sweeps=sweeps, cutoff=cutoff,
                  silent=silent, goal=goal, cvgE=cvgE, SvNbond=SvNbond, noise=noise,
                  noise_goal=noise_goal, noise_incr=noise_incr, halfsweep=halfsweep, kwargs...)
  end
  dmrg_b200(psi, mpo; maxm=maxm, minm=minm, sweeps=sweeps, cutoff=cutoff, silent=silent,
            goal=goal, cvgE=cvgE, SvNbond=SvNbond, krylov=krylov, precision=precision,
            charges=charges, device=device, method=method, noise=Float64(noise),
            noise_goal=noise_goal, noise_incr=noise_incr, halfsweep=halfsweep)
end

"""
    dmrg_b200(psi, mpo; maxm, minm=2, sweeps=1, cutoff=0.0, silent=false, goal=0.0, cvgE=true,
              SvNbond=0, krylov=2, precision=0, charges=nothing, device=0, method="twosite",
              noise=1.0, noise_goal=0.3, noise_incr=0.01)

The GPU DMRG behind the `dmrg` method (two-site, or 3S single-site sweeps with subspace
expansion). Returns the energy of the last bond step and updates `psi` (tensors and `oc`) in
place.
"""
function dmrg_b200(psi, mpo; maxm::Integer=0, minm::Integer=2, sweeps::Integer=1,
                   cutoff::Float64=0.0, silent::Bool=false, goal::Float64=0.0, cvgE::Bool=true,
                   SvNbond::Integer=0, krylov::Integer=2, precision::Integer=0, charges=nothing,
                   device::Integer=0, method::String="twosite", noise::Float64=1.0,
                   noise_goal::Float64=0.3, noise_incr::Float64=0.01, halfsweep::Bool=false)
  ctx = context(device)
  ch = site_charges(psi, charges)
  hmpo = upload_mpo(ctx, mpo, ch)
  st = upload_mps(ctx, hmpo, psi, ch)
  try
    check(ccall((:dmrg_env_build, libdmrg), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), st, hmpo), ctx.h,
          "dmrg_env_build")
    p = Params()
    ccall((:dmrg_params_default, libdmrg), Cvoid, (Ref{Params},), p)
    p.maxm, p.minm, p.cutoff, p.krylov, p.precision, p.svnbond = maxm, minm, cutoff, krylov,
                                                                 precision, SvNbond
    p.goal, p.cvgE = goal, cvgE ? 1 : 0
    p.halfsweep = halfsweep ? 1 : 0
    nz = method == "3S" ? Noise(noise, noise_goal, noise_incr, 0.0) : nothing
    energy = run_sweeps!(ctx, st, hmpo, p, sweeps, silent, nz)
    write_back!(ctx, st, psi, ch)
    return energy
  finally
    ccall((:dmrg_state_destroy, libdmrg), Cint, (Ptr{Cvoid},), st)
    ccall((:dmrg_mpo_destroy, libdmrg), Cint, (Ptr{Cvoid},), hmpo)
  end
end

# ------------------------------------------------------------------------ TDVP

"""
    tdvp_twosite(psi, mpo; m, minm=2, cutoff=0., origj=true, r=2, prefactor=1., precision=0,
                 charges=nothing, device=0)
    tdvp(psi, mpo; ...)

The reference's TDVP calls (algs/time.jl:211-363) on the GPU when `prefactor` is real and the
tensors are real: one half sweep of steps, each propagator exp(tau H) applied by a Krylov
exponential with `r` vectors. Returns En of the last Krylov call and updates `psi` in place. A
complex prefactor (real-time evolution) or complex tensors run the reference's own code. The
single-site form stops at the chain's edge after L-1 steps.
"""
function DMRJtensor.tdvp_twosite(psi::DMRJtensor.matrixproductstate,
                                 mpo::DMRJtensor.matrixproductoperator;
                                 m::Integer=maximum([size(psi[w], 3) for w = 1:length(psi)]),
                                 minm::Integer=2, cutoff::Real=0., origj::Bool=true,
                                 r::Integer=2, prefactor::Number=1., precision::Integer=0,
                                 charges=nothing, device::Integer=0)
  if !gpu_tdvp_ok(psi, prefactor, origj)
    return invoke(DMRJtensor.tdvp_twosite, Tuple{DMRJtensor.MPS,DMRJtensor.MPO}, psi, mpo;
                  m=m, minm=minm, cutoff=cutoff, origj=origj, r=r, prefactor=prefactor)
  end
  tdvp_b200(psi, mpo, true; m=m, minm=minm, cutoff=Float64(cutoff), r=r,
            prefactor=Float64(real(prefactor)), precision=precision, charges=charges,
            device=device)
end

function DMRJtensor.tdvp(psi::DMRJtensor.matrixproductstate, mpo::DMRJtensor.matrixproductoperator;
                         m::Integer=maximum([size(psi[w], 3) for w = 1:length(psi)]),
                         minm::Integer=2, cutoff::Real=0., origj::Bool=true, r::Integer=2,
                         prefactor::Number=1., precision::Integer=0, charges=nothing,
                         device::Integer=0)
  if !gpu_tdvp_ok(psi, prefactor, origj)
    return invoke(DMRJtensor.tdvp, Tuple{DMRJtensor.MPS,DMRJtensor.MPO}, psi, mpo;
                  m=m, minm=minm, cutoff=cutoff, origj=origj, r=r, prefactor=prefactor)
  end
  tdvp_b200(psi, mpo, false; m=m, minm=minm, cutoff=Float64(cutoff), r=r,
            prefactor=Float64(real(prefactor)), precision=precision, charges=charges,
            device=device)
end

gpu_tdvp_ok(psi, prefactor, origj) =
  imag(prefactor) == 0 && !(eltype(psi.A[1]) <: Complex) &&
  (origj || psi.oc == 1 || psi.oc == length(psi))

function tdvp_b200(psi, mpo, twosite::Bool; m::Integer, minm::Integer=2, cutoff::Float64=0.0,
                   r::Integer=2, prefactor::Float64=1.0, precision::Integer=0, charges=nothing,
                   device::Integer=0)
  ctx = context(device)
  ch = site_charges(psi, charges)
  hmpo = upload_mpo(ctx, mpo, ch)
  st = upload_mps(ctx, hmpo, psi, ch)
  try
    # makeEnv(psi, psi, mpo) at the start of every call (algs/time.jl:214,291)
    check(ccall((:dmrg_env_build, libdmrg), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), st, hmpo), ctx.h,
          "dmrg_env_build")
    p = Params()
    ccall((:dmrg_params_default, libdmrg), Cvoid, (Ref{Params},), p)
    p.maxm, p.minm, p.cutoff, p.krylov, p.precision = m, minm, cutoff, r, precision
    stats = SweepStats()
    check(ccall((:dmrg_tdvp, libdmrg), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Ref{Params}, Cdouble, Cint, Ref{SweepStats}),
                st, hmpo, p, prefactor, twosite ? 1 : 0, stats), ctx.h, "dmrg_tdvp")
    write_back!(ctx, st, psi, ch)
    return stats.energy
  finally
    ccall((:dmrg_state_destroy, libdmrg), Cint, (Ptr{Cvoid},), st)
    ccall((:dmrg_mpo_destroy, libdmrg), Cint, (Ptr{Cvoid},), hmpo)
  end
end

function bond_info(ctx, st, b, nsym)
  n = Ref{Cint}(0)
  check(ccall((:dmrg_bond_info, libdmrg), Cint, (Ptr{Cvoid}, Cint, Ref{Cint}, Ptr{Cint}, Ptr{Cint}),
              st, b, n, C_NULL, C_NULL), ctx.h, "dmrg_bond_info")
  q = zeros(Cint, max(n[] * max(nsym, 1), 1))
  dims = zeros(Cint, max(n[], 1))
  check(ccall((:dmrg_bond_info, libdmrg), Cint, (Ptr{Cvoid}, Cint, Ref{Cint}, Ptr{Cint}, Ptr{Cint}),
              st, b, n, q, dims), ctx.h, "dmrg_bond_info")
  ([Int.(q[(k - 1) * nsym + 1:k * nsym]) for k = 1:n[]], Int.(dims[1:n[]]))
end

# Writes the device MPS back into psi, one site at a time. Dense states receive the
# dense-equivalent array; quantum-number states a Qtens built from it with the bond labels the
# library reports (the bond bases grouped by charge: a gauge change of the same state), as
# makeqMPS does (lib/MPS/makeqMPS.jl:40-64).
function write_back!(ctx::Context, st, psi, ch)
  L = length(psi.A)
  qn = ch !== nothing && isqtens(psi.A[1])
  nsym = qn ? size(ch[1], 2) : 0
  Q = qn ? typeof(DMRJtensor.getQnum(2, 1, psi.A[1])) : Nothing
  qlab(b) = begin
    qs, dims = bond_info(ctx, st, b, nsym)
    [Q(q...) for (q, dd) in zip(qs, dims) for _ = 1:dd]
  end
  left = qn ? qlab(0) : nothing
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
    if qn
      right = qlab(i)
      phys = [DMRJtensor.getQnum(2, s, psi.A[i]) for s = 1:d]
      psi.A[i] = DMRJtensor.Qtens(A, [left, phys, inv.(right)])
      left = right
    else
      psi.A[i] = DMRJtensor.convertTens(eltype(psi.A), A)
    end
  end
  oc = Ref{Cint}(0)
  check(ccall((:dmrg_state_oc, libdmrg), Cint, (Ptr{Cvoid}, Ref{Cint}), st, oc), ctx.h, "dmrg_state_oc")
  psi.oc = oc[] + 1
  psi
end

# ------------------------------------------------------------------------ the Env API

"""
    B200Env, B200Side

Resident environments of one (psi, mpo) pair on the GPU. `Lenv, Renv = makeEnv_b200(psi, mpo)`
builds them (makeEnv, lib/Env/makeEnv.jl:196-221); `Lenv[i]` / `Renv[i]` download the
dense-equivalent [m, w, m] tensors (L[bra, w, ket], R[ket, w, bra]); `Lupdate!(i, Lenv, psi, mpo)`
and `Rupdate!(i, Renv, psi, mpo)` are the reference's in-place updates (lib/MPO_MPS/Lupdate.jl:34,
Rupdate.jl:34) on the device, with the state's own site tensors.
"""
mutable struct B200Env
  ctx::Context
  mpo::Ptr{Cvoid}
  st::Ptr{Cvoid}
  L::Int
end

struct B200Side
  env::B200Env
  left::Bool
end

function makeEnv_b200(psi, mpo; charges=nothing, device::Integer=0)
  ctx = context(device)
  ch = site_charges(psi, charges)
  hmpo = upload_mpo(ctx, mpo, ch)
  st = upload_mps(ctx, hmpo, psi, ch)
  check(ccall((:dmrg_env_build, libdmrg), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), st, hmpo), ctx.h, "dmrg_env_build")
  e = B200Env(ctx, hmpo, st, length(psi.A))
  finalizer(e) do x
    ccall((:dmrg_state_destroy, libdmrg), Cint, (Ptr{Cvoid},), x.st)
    ccall((:dmrg_mpo_destroy, libdmrg), Cint, (Ptr{Cvoid},), x.mpo)
  end
  (B200Side(e, true), B200Side(e, false))
end

Base.length(s::B200Side) = s.env.L

function Base.getindex(s::B200Side, i::Integer)
  e = s.env
  dims = zeros(Cint, 3)
  check(ccall((:dmrg_env_get, libdmrg), Cint, (Ptr{Cvoid}, Cint, Cint, Ptr{Cdouble}, Ptr{Cint}),
              e.st, i - 1, s.left ? 1 : 0, C_NULL, dims), e.ctx.h, "dmrg_env_get (sizes)")
  out = Array{Float64}(undef, dims...)
  check(ccall((:dmrg_env_get, libdmrg), Cint, (Ptr{Cvoid}, Cint, Cint, Ptr{Cdouble}, Ptr{Cint}),
              e.st, i - 1, s.left ? 1 : 0, out, dims), e.ctx.h, "dmrg_env_get")
  out
end

function DMRJtensor.Lupdate!(i::Integer, Lenv::B200Side, psi::DMRJtensor.MPS, mpo::DMRJtensor.MPO...)
  Lenv.left || error("Lupdate! needs the left environment list")
  check(ccall((:dmrg_lupdate, libdmrg), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Cint), Lenv.env.st,
              Lenv.env.mpo, i - 1), Lenv.env.ctx.h, "dmrg_lupdate")
  nothing
end

function DMRJtensor.Rupdate!(i::Integer, Renv::B200Side, psi::DMRJtensor.MPS, mpo::DMRJtensor.MPO...)
  Renv.left && error("Rupdate! needs the right environment list")
  check(ccall((:dmrg_rupdate, libdmrg), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Cint), Renv.env.st,
              Renv.env.mpo, i - 1), Renv.env.ctx.h, "dmrg_rupdate")
  nothing
end

# Lupdate(Lenv, dualpsi, psi, mpo) / Rupdate(Renv, dualpsi, psi, mpo) (lib/MPO_MPS/Lupdate.jl:17,
# Rupdate.jl:17) on dense Float64 arrays, computed on the device (dmrg_env_step).
function env_step(left::Bool, E::Array{Float64,3}, dual::Array{Float64,3}, psi::Array{Float64,3},
                  W::Array{Float64,4}; device::Integer=0)
  ctx = context(device)
  ml, d, mr = size(psi)
  wl, wr = size(W, 1), size(W, 4)
  out = Array{Float64}(undef, left ? (mr, wr, mr) : (ml, wl, ml))
  check(ccall((:dmrg_env_step, libdmrg), Cint,
              (Ptr{Cvoid}, Cint, Cint, Cint, Cint, Cint, Cint, Ptr{Cdouble}, Ptr{Cdouble},
               Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}),
              ctx.h, left ? 1 : 0, ml, d, mr, wl, wr, E, dual, psi, W, out), ctx.h, "dmrg_env_step")
  out
end

DMRJtensor.Lupdate(L::Array{Float64,3}, dual::Array{Float64,3}, psi::Array{Float64,3},
                   W::Array{Float64,4}) = env_step(true, L, dual, psi, W)
DMRJtensor.Rupdate(R::Array{Float64,3}, dual::Array{Float64,3}, psi::Array{Float64,3},
                   W::Array{Float64,4}) = env_step(false, R, dual, psi, W)

# expect(psi, H) (lib/MPO_MPS/expect.jl:47-56) on the state of a device environment pair:
# <psi|H|psi>, not normalised; `H` is another uploaded MPO over the same sites (default: its own).
function expect_b200(s::B200Side, hmpo::Ptr{Cvoid}=s.env.mpo)
  v = Ref{Cdouble}(0.0)
  check(ccall((:dmrg_expect, libdmrg), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Ref{Cdouble}), s.env.st,
              hmpo, v), s.env.ctx.h, "dmrg_expect")
  v[]
end

# correlationmatrix(psi, Cc, Ca; trail) (lib/MPO_MPS/correlationmatrix.jl:21-83), operators
# O[bra, ket] as d x d Float64 matrices; the centre of the state is not moved.
function correlationmatrix_b200(s::B200Side, Cc::Matrix{Float64}, Ca::Matrix{Float64};
                                trail=nothing)
  d = size(Cc, 1)
  L = s.env.L
  rho = Matrix{Float64}(undef, L, L)
  F = trail === nothing ? C_NULL : Matrix{Float64}(trail)
  check(ccall((:dmrg_correlationmatrix, libdmrg), Cint,
              (Ptr{Cvoid}, Cint, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}),
              s.env.st, d, Cc, Ca, F, rho), s.env.ctx.h, "dmrg_correlationmatrix")
  rho
end

# correlation(psi, ops...; sites, trail) (lib/MPO_MPS/correlation.jl:73-237) with dualpsi = psi:
# each operator a d x d Float64 matrix O[bra, ket] or a vector of them on consecutive sites,
# `sites` 1-based start ranges (default 1:L), `trail` one matrix, a tuple of them, or ().
function correlation_b200(s::B200Side, ops...; sites=ntuple(i -> 1:s.env.L, length(ops)),
                          trail=())
  n = length(ops)
  fs = [o isa AbstractVector ? collect(o) : [o] for o in ops]
  lens = Cint[length(f) for f in fs]
  d = size(fs[1][1], 1)
  opbuf = reduce(vcat, [vec(Matrix{Float64}(m)) for f in fs for m in f])
  starts = [Cint[x - 1 for x in sq] for sq in sites]
  base = [length(starts[g]) - (lens[g] - 1) for g = 1:n]
  tl = trail isa Tuple ? collect(trail) : (trail isa AbstractMatrix ? [trail] : collect(trail))
  tb = isempty(tl) ? C_NULL : reduce(vcat, [vec(Matrix{Float64}(tl[(g - 1) % length(tl) + 1]))
                                            for g = 1:n])
  omega = zeros(Float64, base...)
  check(ccall((:dmrg_correlation, libdmrg), Cint,
              (Ptr{Cvoid}, Cint, Cint, Ptr{Cint}, Ptr{Cdouble}, Ptr{Cint}, Ptr{Cint}, Ptr{Cdouble},
               Ptr{Cdouble}),
              s.env.st, d, n, lens, opbuf, Cint[length(x) for x in starts], reduce(vcat, starts), tb,
              omega), s.env.ctx.h, "dmrg_correlation")
  omega
end

# Checkpoint of the device state (the persistence of largeMPS / loadMPS,
# lib/MPS/largeMPS.jl:19-81); load_b200 returns a new environment pair, rebuilt.
save_b200(s::B200Side, path::AbstractString) =
  check(ccall((:dmrg_state_save, libdmrg), Cint, (Ptr{Cvoid}, Cstring), s.env.st, path),
        s.env.ctx.h, "dmrg_state_save")

function load_b200(s::B200Side, path::AbstractString)
  e = s.env
  out = Ref{Ptr{Cvoid}}(C_NULL)
  check(ccall((:dmrg_state_load, libdmrg), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Cstring, Ref{Ptr{Cvoid}}),
              e.ctx.h, e.mpo, path, out), e.ctx.h, "dmrg_state_load")
  check(ccall((:dmrg_env_build, libdmrg), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), out[], e.mpo), e.ctx.h,
        "dmrg_env_build")
  ne = B200Env(e.ctx, e.mpo, out[], e.L)   # shares the MPO handle: frees only its state
  finalizer(x -> ccall((:dmrg_state_destroy, libdmrg), Cint, (Ptr{Cvoid},), x.st), ne)
  (B200Side(ne, true), B200Side(ne, false))
end

end # module
