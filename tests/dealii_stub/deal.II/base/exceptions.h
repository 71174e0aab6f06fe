// Stand-in for deal.II/base/exceptions.h: exception base, ExcMessage, AssertThrow and the
// exception-declaration macros MeltPoolDG's core/exceptions.hpp uses.
#pragma once
#include <stdexcept>
#include <string>

namespace dealii
{
  struct ExceptionBase : std::runtime_error
  {
    explicit ExceptionBase(const std::string &what = "deal.II exception")
      : std::runtime_error(what)
    {}
  };
  struct ExcMessage : ExceptionBase
  {
    explicit ExcMessage(const std::string &msg)
      : ExceptionBase(msg)
    {}
  };
} // namespace dealii

#define AssertThrow(cond, exc) \
  do                           \
    {                          \
      if (!(cond))             \
        throw exc;             \
    }                          \
  while (false)
#define Assert(cond, exc) AssertThrow(cond, exc)
#define DEAL_II_NOT_IMPLEMENTED() throw ::dealii::ExcMessage("not implemented")
#define DeclExceptionMsg(Name, msg)                 \
  struct Name : ::dealii::ExceptionBase             \
  {                                                 \
    Name()                                          \
      : ::dealii::ExceptionBase(msg)                \
    {}                                              \
  }
#define DeclException1(Name, T1, out)                                \
  struct Name : ::dealii::ExceptionBase                              \
  {                                                                  \
    explicit Name(const T1 &)                                        \
    {}                                                               \
  }
#define DeclException2(Name, T1, T2, out)                            \
  struct Name : ::dealii::ExceptionBase                              \
  {                                                                  \
    Name(const T1 &, const T2 &)                                     \
    {}                                                               \
  }
