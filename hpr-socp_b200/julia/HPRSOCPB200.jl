# HPRSOCPB200.jl — Julia binding of libhprsocp_b200.so.
#
# Drop-in for the GPU solve of PolyU-IOR/HPR-SOCP: `optimize(model, params)`
# takes the reference's own `QP_info_cpu` and `HPRSOCP_parameters`
# (src/structs.jl:127-150, 251-277) and returns its `HPRSOCP_results`
# (src/structs.jl:297-314), running every vector operation of `solve`
# (src/algorithm.jl:2765-2905) inside the shared library through `ccall`.
# The reference package includes this file and routes `optimize`
# (src/algorithm.jl:2538-2581) here; the MOI wrapper (MOI_wrapper.jl:683-693)
# then uses it unchanged.
#
# The caller's arrays are copied to the device once per solve.  A is passed
# as CSR through the CSC storage of A' (QP_info_cpu.AT): colptr, rowval and
# nzval of A' are the 1-based row pointers, column indices and values of A.
module HPRSOCPB200

using SparseArrays

const LIB = Ref{String}(joinpath(@__DIR__, "..", "lib", "libhprsocp_b200.so"))

const HPR_Q_NONE = Int32(0)
const HPR_Q_CSR = Int32(1)
const HPR_Q_DIAG_LOWRANK = Int32(2)
const HPR_Q_OPERATOR = Int32(3)

const BC_NORM = Dict(:l2 => Int32(0), :rms => Int32(1), :linf => Int32(2), :l_inf => Int32(2), :inf => Int32(2))
const SOC_STRATEGY = Dict(
    :max => 1, :rms => 2, :geom => 3, :adaptive => 4, :hybrid => 5, :ruiz_geom => 6,
    :role_split => 7, :pock_safe_role_split => 8, :size_split_role_split => 9,
    :pre_pock_size_split => 10, :pre_pock_huge_var_taper => 11,
    :pre_pock_huge_var_taper_pock_geom => 12, :pre_pock_band_split => 13,
    :pre_pock_constraint_rms => 14, :pre_pock_constraint_max => 15,
    :pre_pock_constraint_taper => 16, :small_cone_constraint_max => 17,
    :count_aware_small_cone_bias => 18, :phase_blend => 19, :phase_taper => 20)
const STATUS = ("OPTIMAL", "MAX_ITER", "TIME_LIMIT")

# ---- C structs (include/hprsocp_b200.h), field for field ----------------
struct CCSR
    nrows::Int64
    ncols::Int64
    nnz::Int64
    rowptr::Ptr{Int32}
    colind::Ptr{Int32}
    values::Ptr{Float64}
end
CCSR() = CCSR(0, 0, 0, C_NULL, C_NULL, C_NULL)

struct CProblem
    m::Int64
    n::Int64
    m_lin::Int64
    n_box::Int64
    A::CCSR
    AT::CCSR
    c::Ptr{Float64}
    l::Ptr{Float64}
    u::Ptr{Float64}
    AL::Ptr{Float64}
    AU::Ptr{Float64}
    soc_rhs::Ptr{Float64}
    soc_con_idx::Ptr{Int64}
    n_soc_con_idx::Int64
    soc_var_idx::Ptr{Int64}
    n_soc_var_idx::Int64
    index_base::Int32
    q_kind::Int32
    Q::CCSR
    q_diag::Ptr{Float64}
    F::CCSR
    obj_constant::Float64
end

struct CParams
    stoptol::Float64
    sigma::Float64
    max_iter::Int64
    time_limit::Float64
    check_iter::Int64
    print_frequency::Int64
    device_number::Int32
    use_Ruiz_scaling::Int32
    ruiz_iterations::Int32
    use_bc_scaling::Int32
    bc_scaling_norm_type::Int32
    use_Pock_Chambolle_scaling::Int32
    soc_block_scaling_strategy::Int32
    verbose::Int32
    initial_x::Ptr{Float64}
    initial_y::Ptr{Float64}
    lambda_max_A::Float64
    lambda_max_Q::Float64
    precision::Int32
    refine::Int32
    auto_save::Int32
    save_filename::Ptr{UInt8}
end

struct CResiduals
    err_Rp_org_bar::Float64
    err_Rp_linear_org_bar::Float64
    err_Rp_soc_org_bar::Float64
    err_Rd_org_bar::Float64
    KKTx_and_gap_org_bar::Float64
    primal_obj_bar::Float64
    rel_gap_bar::Float64
    dual_obj_bar::Float64
end

mutable struct CResults
    iter::Int64
    iter_4::Int64
    iter_6::Int64
    time::Float64
    time_4::Float64
    time_6::Float64
    power_time::Float64
    primal_obj::Float64
    residuals::Float64
    gap::Float64
    status::Int32
    restarts::Int32
    sigma_final::Float64
    lambda_max_A::Float64
    lambda_max_Q::Float64
    last::CResiduals
    x::Ptr{Float64}
    y::Ptr{Float64}
    z::Ptr{Float64}
    w::Ptr{Float64}
end
CResults() = CResults(0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                      CResiduals(0, 0, 0, 0, 0, 0, 0, 0), C_NULL, C_NULL, C_NULL, C_NULL)

struct CCbfData
    m::Int64
    n::Int64
    number_eq::Int64
    number_ineq::Int64
    A::CCSR
    rhs::Ptr{Float64}
    c::Ptr{Float64}
    l::Ptr{Float64}
    u::Ptr{Float64}
    soc_con_idx::Ptr{Int64}
    n_soc_con_idx::Int64
    soc_var_idx::Ptr{Int64}
    n_soc_var_idx::Int64
    obj_constant::Float64
end

"""Diagonal-plus-low-rank quadratic term Q = Diagonal(d) + F'F, applied as an
operator (the form the library's Q operator supports besides a CSR Q)."""
struct DiagPlusLowRankQ
    d::Vector{Float64}
    F::SparseMatrixCSC{Float64,Int}
end

# CSR view of M built from the CSC storage of M' (1-based); `keep` holds the
# converted arrays until the call returns.
function csr_of_transpose(Mt::SparseMatrixCSC, nrows::Integer, ncols::Integer, keep::Vector{Any})
    rp = Int32.(Mt.colptr)
    ci = Int32.(Mt.rowval)
    v = Vector{Float64}(Mt.nzval)
    push!(keep, rp, ci, v)
    return CCSR(nrows, ncols, length(v), pointer(rp), pointer(ci), pointer(v))
end

function c_params(params, keep::Vector{Any})
    x0 = params.initial_x === nothing ? C_NULL : pointer(push!(keep, Vector{Float64}(params.initial_x))[end])
    y0 = params.initial_y === nothing ? C_NULL : pointer(push!(keep, Vector{Float64}(params.initial_y))[end])
    haskey(BC_NORM, params.bc_scaling_norm_type) ||
        error("Unsupported bc scaling norm_type: $(params.bc_scaling_norm_type). Use :l2, :rms, or :linf.")
    haskey(SOC_STRATEGY, params.soc_block_scaling_strategy) ||
        error("Unsupported soc_block_scaling_strategy=$(params.soc_block_scaling_strategy).")
    precision = hasproperty(params, :precision) ? Int32(params.precision) : Int32(0)
    refine = hasproperty(params, :refine) ? Int32(params.refine) : Int32(0)
    # the auto-save archive is .npz (member names = the reference's HDF5
    # paths); the reference's default name "….h5" is mapped to "….npz"
    fname = endswith(params.save_filename, ".h5") ? params.save_filename[1:end-3] * ".npz" : params.save_filename
    fbytes = push!(Vector{UInt8}(codeunits(fname)), 0x00)
    push!(keep, fbytes)
    return CParams(params.stoptol, params.sigma, params.max_iter, params.time_limit, params.check_iter,
                   params.print_frequency, Int32(params.device_number), Int32(params.use_Ruiz_scaling),
                   Int32(params.ruiz_iterations), Int32(params.use_bc_scaling),
                   BC_NORM[params.bc_scaling_norm_type], Int32(params.use_Pock_Chambolle_scaling),
                   Int32(SOC_STRATEGY[params.soc_block_scaling_strategy]), Int32(params.verbose), x0, y0,
                   -1.0, -1.0, precision, refine, Int32(params.auto_save), pointer(fbytes))
end

function c_problem(model, keep::Vector{Any})
    m, n = size(model.A)
    A = csr_of_transpose(model.AT, m, n, keep)          # CSC(A') == CSR(A)
    AT = csr_of_transpose(model.A, n, m, keep)          # CSC(A)  == CSR(A')
    vecs = map(v -> pointer(push!(keep, Vector{Float64}(v))[end]),
               (model.c, model.l, model.u, model.AL, model.AU, model.soc_rhs))
    con = push!(keep, Vector{Int64}(model.SOC_con_idx))[end]
    var = push!(keep, Vector{Int64}(model.SOC_var_idx))[end]
    qkind, Q, qd, F = HPR_Q_NONE, CCSR(), Ptr{Float64}(C_NULL), CCSR()
    if model.Q isa SparseMatrixCSC
        if nnz(model.Q) > 0
            qkind = HPR_Q_CSR
            Q = csr_of_transpose(model.Q, n, n, keep)   # Q is symmetric
        end
    elseif model.Q isa DiagPlusLowRankQ
        qkind = HPR_Q_DIAG_LOWRANK
        qd = pointer(push!(keep, Vector{Float64}(model.Q.d))[end])
        k = size(model.Q.F, 1)
        F = csr_of_transpose(sparse(transpose(model.Q.F)), k, n, keep)
    elseif model.Q !== nothing && !is_user_operator(model.Q)
        error("HPRSOCPB200 supports a sparse Q, DiagPlusLowRankQ or a user Q operator, got $(typeof(model.Q))")
    end
    return CProblem(m, n, model.number_linear_con, model.number_lu_x, A, AT, vecs..., pointer(con), length(con),
                    pointer(var), length(var), Int32(1), qkind, Q, qd, F, model.obj_constant)
end

# ---- a user Q operator (src/Q_operators/Q_operator_interface.jl:32-151) ---
# A model whose Q is a user AbstractQOperatorCPU keeps q_kind NONE in the
# upload; the library then calls back into Julia for every product Q v
# (hpr_set_q_operator).  The callback views the library's device vectors as
# CuArrays (CUDA.jl, loaded by the caller) and runs the operator's GPU form,
# made once by the reference's to_gpu, through its Qmap!(x, Qx, Q), on the
# stream the library passes in.
is_user_operator(Q) = isdefined(Main, :HPRSOCP) && Q isa Main.HPRSOCP.AbstractQOperatorCPU

struct QOperatorBox
    gpu::Any  # the operator's GPU form (to_gpu)
end

function q_apply(user::Ptr{Cvoid}, vin::Ptr{Float64}, vout::Ptr{Float64}, n::Int64, stream::Ptr{Cvoid})::Cvoid
    box = unsafe_pointer_to_objref(user)::QOperatorBox
    CUDA = Main.CUDA
    x = unsafe_wrap(CUDA.CuArray, CUDA.CuPtr{Float64}(UInt(vin)), Int(n); own = false)
    Qx = unsafe_wrap(CUDA.CuArray, CUDA.CuPtr{Float64}(UInt(vout)), Int(n); own = false)
    CUDA.stream!(CUDA.CuStream(reinterpret(CUDA.CUstream, stream))) do
        Main.HPRSOCP.Qmap!(x, Qx, box.gpu)
    end
    return nothing
end

function check(rc::Integer)
    rc == 0 && return
    msg = unsafe_string(ccall((:hpr_status_string, LIB[]), Cstring, (Cint,), rc))
    error("libhprsocp_b200: $msg")
end

"""
    optimize(model::QP_info_cpu, params::HPRSOCP_parameters, Results::Type)

Solve on one B200 and return `Results(...)` (the reference's
`HPRSOCP_results`).  `params.use_gpu == false` is an error: there is no CPU
fallback.  `params.warm_up` is ignored (the kernels are compiled ahead of
time).
"""
function optimize(model, params, Results::Type)
    params.use_gpu || error("HPRSOCPB200 has no CPU path: set use_gpu = true")
    keep = Any[]
    prob = c_problem(model, keep)
    p = c_params(params, keep)
    m, n = size(model.A)
    x, y, z, w = zeros(n), zeros(m), zeros(n), zeros(n)
    res = CResults()
    res.x, res.y, res.z, res.w = pointer(x), pointer(y), pointer(z), pointer(w)
    if model.Q !== nothing && is_user_operator(model.Q)
        # context, upload, the operator, solve (hpr_optimize has no operator)
        box = QOperatorBox(Main.HPRSOCP.to_gpu(model.Q))
        fn = @cfunction(q_apply, Cvoid, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Int64, Ptr{Cvoid}))
        h = Ref{Ptr{Cvoid}}(C_NULL)
        check(ccall((:hpr_create, LIB[]), Cint, (Cint, Csize_t, Ref{Ptr{Cvoid}}), Cint(params.device_number), 0, h))
        try
            GC.@preserve keep x y z w box begin
                check(ccall((:hpr_upload, LIB[]), Cint, (Ptr{Cvoid}, Ref{CProblem}), h[], prob))
                check(ccall((:hpr_set_q_operator, LIB[]), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Any, Cdouble), h[], fn, box,
                            0.0))
                check(ccall((:hpr_solve, LIB[]), Cint, (Ptr{Cvoid}, Ref{CParams}, Ref{CResults}), h[], p, res))
            end
        finally
            ccall((:hpr_destroy, LIB[]), Cint, (Ptr{Cvoid},), h[])
        end
    else
        GC.@preserve keep x y z w begin
            rc = ccall((:hpr_optimize, LIB[]), Cint, (Ref{CProblem}, Ref{CParams}, Ref{CResults}), prob, p, res)
        end
        check(rc)
    end
    out = Results()
    out.iter, out.iter_4, out.iter_6 = res.iter, res.iter_4, res.iter_6
    out.time, out.time_4, out.time_6, out.power_time = res.time, res.time_4, res.time_6, res.power_time
    out.primal_obj, out.residuals, out.gap = res.primal_obj, res.residuals, res.gap
    out.status = STATUS[res.status + 1]
    out.x, out.y, out.z, out.w = x, y, z, w
    return out
end

"""
    read_cbf(filename; threads = 0)

The reference's `read_cbf` (src/utils/cbf_io.jl:1438-1455) run by the
library's multi-threaded C++ reader (`hpr_cbf_read`).  Returns the same
values: `(Q, c, A, b, SOC_con_idx, number_eq, number_ineq, lb, ub,
SOC_var_idx, obj_constant)` with `A::SparseMatrixCSC{Float64,Int32}`, ready
for the reference's `build_from_SOCP_data`.
"""
function read_cbf(filename::AbstractString; threads::Integer = 0)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    rc = ccall((:hpr_cbf_read, LIB[]), Cint, (Cstring, Cint, Ref{Ptr{Cvoid}}), filename, Cint(threads), h)
    rc == 0 || error(unsafe_string(ccall((:hpr_cbf_last_error, LIB[]), Cstring, ())))
    try
        d = Ref{CCbfData}()
        check(ccall((:hpr_cbf_data_get, LIB[]), Cint, (Ptr{Cvoid}, Ref{CCbfData}), h[], d))
        D = d[]
        copyv(p::Ptr{T}, k) where {T} = k == 0 ? T[] : copy(unsafe_wrap(Array, p, Int(k)))
        m, n, nz = Int(D.m), Int(D.n), Int(D.A.nnz)
        # the CSR arrays of A are the CSC arrays of A' (0-based -> 1-based)
        At = SparseMatrixCSC{Float64,Int32}(n, m, copyv(D.A.rowptr, m + 1) .+ Int32(1),
                                            copyv(D.A.colind, nz) .+ Int32(1), copyv(D.A.values, nz))
        A = copy(transpose(At))
        return (spzeros(Float64, n, n), copyv(D.c, n), A, copyv(D.rhs, m),
                Vector{Int}(copyv(D.soc_con_idx, D.n_soc_con_idx)), Int(D.number_eq), Int(D.number_ineq),
                copyv(D.l, n), copyv(D.u, n), Vector{Int}(copyv(D.soc_var_idx, D.n_soc_var_idx)), D.obj_constant)
    finally
        ccall((:hpr_cbf_free, LIB[]), Cvoid, (Ptr{Cvoid},), h[])
    end
end

end # module
