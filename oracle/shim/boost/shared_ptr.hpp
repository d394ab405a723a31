// Stand-in for boost::shared_ptr (the reference Tensor's ref-count holder).
#pragma once
#include <memory>
namespace boost { using std::shared_ptr; }
