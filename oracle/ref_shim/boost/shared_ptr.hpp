// boost::shared_ptr as std::shared_ptr.
#pragma once
#include <memory>
namespace boost {
using std::shared_ptr;
}
