// The plan interface of the hptt C++ API (B200 build).
//
// CGraphTransPackBase<T> keeps the reference's virtual interface
// (inc/hptt/impl/hptt_trans.h:12-36): exec / operator() / print_plan /
// reset_data / set_thread_ids / unset_thread_ids, non-copyable, non-movable,
// with trans_plan<T> as its alias.  On the GPU:
//   exec()           enqueues the transpose on the plan's CUDA stream and
//                    returns; results are visible after sync() (or any
//                    later stream-ordered work).  Like the reference it
//                    returns nothing: a launch error is kept and read back
//                    with status().
//   set_thread_ids   accepted and ignored (there is no host thread team).
// The GPU-only calls (sync, set_stream, exec_on, status, set_coef) are
// extensions, declared on CudaTransPlan<T> below; create_plan returns a plan
// that is one, so std::dynamic_pointer_cast reaches them.
#pragma once
#ifndef HPTT_IMPL_HPTT_TRANS_H_
#define HPTT_IMPL_HPTT_TRANS_H_

#include <cstdint>
#include <string>
#include <vector>

#include <hptt/types.h>

namespace hptt {

template <typename FloatType>
class CGraphTransPackBase {
 public:
  CGraphTransPackBase() = default;
  CGraphTransPackBase(const CGraphTransPackBase &) = delete;
  CGraphTransPackBase &operator=(const CGraphTransPackBase &) = delete;
  CGraphTransPackBase(CGraphTransPackBase &&) = delete;
  CGraphTransPackBase &operator=(CGraphTransPackBase &&) = delete;
  virtual ~CGraphTransPackBase() = default;

  virtual void exec() = 0;
  virtual void operator()() = 0;
  virtual void print_plan() = 0;
  virtual void reset_data(const FloatType *in_data, FloatType *out_data) = 0;
  virtual void set_thread_ids(const std::vector<int32_t> &thread_ids) = 0;
  virtual void unset_thread_ids() = 0;
};

template <typename FloatType>
using trans_plan = CGraphTransPackBase<FloatType>;

// GPU extensions of a plan.  Every call returns the C ABI status
// (HPTT_OK = 0, codes in hptt_cuda.h).
template <typename FloatType>
class CudaTransPlan : public CGraphTransPackBase<FloatType> {
 public:
  // Wait until every exec enqueued on the plan's stream has finished.
  virtual int sync() = 0;
  // Stream (cudaStream_t passed as void*) used by exec(); nullptr = the
  // legacy default stream, the initial setting.
  virtual int set_stream(void *stream) = 0;
  // Enqueue on an explicit stream.
  virtual int exec_on(void *stream) = 0;
  // Status of the last exec / exec_on (HPTT_OK when it was enqueued).
  virtual int status() const = 0;
  // New real scalars (re-decides whether B is read).
  virtual int set_coef(DeducedFloatType<FloatType> alpha,
                       DeducedFloatType<FloatType> beta) = 0;
  // The summary print_plan() writes.
  virtual std::string describe() const = 0;
  // Algorithmic bytes of one exec: 2*N*sizeof(T), plus N*sizeof(T) when B is read.
  virtual uint64_t bytes() const = 0;
};

}  // namespace hptt

#endif  // HPTT_IMPL_HPTT_TRANS_H_
