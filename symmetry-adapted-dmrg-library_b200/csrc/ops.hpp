// ops.hpp -- the reference's BlockTensor operations, lowered to device task lists.
//
// Each function restates the block-matching loop of the reference method it
// names (file:line given at the definition) on host metadata, and emits the
// dense sector products to the grouped GEMM executor.  Output structures,
// block presence, matching rules and SU(2) factors follow the reference, so a
// tensor produced here has the same blocks as the reference's.
#pragma once
#include "tensor.hpp"

namespace sadmrg {
namespace ops {

template <class S> BTensor<S> fuse(Ctx& c, const Bond& b1, const Bond& b2);
template <class S> BTensor<S> fuse_to_singlet(Ctx& c, const Bond& b1, const Bond& b2);
template <class S> BTensor<S> overlap_initial(Ctx& c, const BTensor<S>& uu, const BTensor<S>& vv, int flag);
template <class S>
BTensor<S> overlap_transformation(Ctx& c, const BTensor<S>& uu, const BTensor<S>& vv, const BTensor<S>& op, int flag);
template <class S>
BTensor<S> operator_initial(Ctx& c, const BTensor<S>& uu, const BTensor<S>& vv, const BTensor<S>& op, int flag);
template <class S>
BTensor<S> operator_transformation(Ctx& c, const BTensor<S>& uu, const BTensor<S>& vv, const BTensor<S>& op, int flag);
template <class S>
BTensor<S> operator_pairup(Ctx& c, const BTensor<S>& uu, const BTensor<S>& vv, const BTensor<S>& op1,
                           const BTensor<S>& op2, int flag);
template <class S> BTensor<S> contract(Ctx& c, const BTensor<S>& t1, int i1, const BTensor<S>& t2, int i2);
// leg permutation of a 3-leg tensor: leg k of the result is leg p[k] of t, the
// bonds moving with their directions (BlockTensor::shift / exchangeindex,
// src/block_tensor_inst.cpp:913-990; for SU(2) the CGC blocks the reference moves
// along are implied by the permuted bonds)
template <class S> BTensor<S> permute3(Ctx& c, const BTensor<S>& t, const int p[3]);

// dst = dst (+) alpha * src with the reference's operator+= presence rules
template <class S> void add_into(Ctx& c, BTensor<S>& dst, const BTensor<S>& src, S alpha);
// U(1) only: dst += chan_w[(q + 2) / 2] * (the blocks of src whose channel leg, bond 1, has charge q)
template <class S> void add_into_channels(Ctx& c, BTensor<S>& dst, const BTensor<S>& src, const S chan_w[3]);
template <class S> void scale(Ctx& c, BTensor<S>& t, S alpha);
template <class S> void take_conjugate(BTensor<S>& t, int bond);
template <class S> void makeup_input_vector(Ctx& c, BTensor<S>& t);
template <class S> void left2right_vectran(Ctx& c, BTensor<S>& t);
template <class S> void right2left_vectran(Ctx& c, BTensor<S>& t);
// host -> device upload of a tensor whose data is given in block order
template <class S> BTensor<S> from_host(Ctx& c, const Struct& st, const std::vector<char>& present, const S* data);
template <class S> std::vector<S> to_host(Ctx& c, const BTensor<S>& t);

// H_eff * psi for one pair term (BlockTensor::hamiltonian_vector_multiplication)
// emitted into an existing plan; see heff.cpp.
struct HvmBufs {
  int psi = 0, out = 1, ops = 2, scratch = 3;
};

}  // namespace ops
}  // namespace sadmrg
