// The boost::mutex / condition_variable surface the reference's pipes use,
// over the standard library.
#pragma once
#include <condition_variable>
#include <mutex>
#include <thread>

// The real header reaches boost/scoped_array.hpp through its own includes;
// wtacpu.cpp relies on that.
#include <boost/scoped_array.hpp>
namespace boost {
struct mutex : std::mutex {
    typedef std::unique_lock<std::mutex> scoped_lock;
};
typedef std::condition_variable condition_variable;
typedef std::thread thread;
}  // namespace boost
