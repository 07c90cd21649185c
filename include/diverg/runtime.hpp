/**
 *  @file  diverg/runtime.hpp
 *  @brief Runtime of the B200 path: the process-wide device context.
 *
 *  Same interface as the reference's include/diverg/runtime.hpp:22-53
 *  (is_runtime_initialized, initialize_runtime, finalize_runtime,
 *  ScopedRuntime).  Where the reference brings up Kokkos, this brings up one
 *  dvg_context (CUDA device, stream and allocator) through the C ABI of
 *  include/dvg.h.  Header-only; link with libdvg.so.
 */
#ifndef DIVERG_B200_RUNTIME_HPP__
#define DIVERG_B200_RUNTIME_HPP__

#include <cstdlib>
#include <mutex>
#include <stdexcept>
#include <string>

#include <dvg.h>

namespace diverg {
  namespace detail {
    struct RuntimeState {
      std::mutex mu;
      dvg_context* ctx = nullptr;
    };

    inline RuntimeState&
    runtime_state( )
    {
      static RuntimeState state;
      return state;
    }

    /** Throws std::runtime_error (the reference's exception type) on failure. */
    inline void
    check( dvg_status s )
    {
      if ( s != DVG_OK ) {
        throw std::runtime_error( std::string( "diverg: " ) + dvg_status_string( s ) + ": "
                                  + dvg_last_error() );
      }
    }

    /** The device ordinal: $DIVERG_DEVICE, else 0. */
    inline int
    default_device( )
    {
      const char* env = std::getenv( "DIVERG_DEVICE" );
      return env ? std::atoi( env ) : 0;
    }
  }  // namespace detail

  /** runtime.hpp:25 */
  inline bool
  is_runtime_initialized( ) noexcept
  {
    auto& st = detail::runtime_state();
    std::lock_guard< std::mutex > lk( st.mu );
    return st.ctx != nullptr;
  }

  /** runtime.hpp:30: initialise the runtime (if not initialised). */
  inline void
  initialize_runtime( )
  {
    auto& st = detail::runtime_state();
    std::lock_guard< std::mutex > lk( st.mu );
    if ( !st.ctx ) detail::check( dvg_init( detail::default_device(), &st.ctx ) );
  }

  /** runtime.hpp:35: finalise the runtime (if it is initialised). */
  inline void
  finalize_runtime( )
  {
    auto& st = detail::runtime_state();
    std::lock_guard< std::mutex > lk( st.mu );
    if ( st.ctx ) {
      dvg_context* c = st.ctx;
      st.ctx = nullptr;
      detail::check( dvg_shutdown( c ) );
    }
  }

  /** runtime.hpp:42-53: RAII guard. */
  class ScopedRuntime {
  public:
    explicit ScopedRuntime( bool finalize_on_destroy = true ) : m_finalize( finalize_on_destroy )
    {
      initialize_runtime();
    }
    ~ScopedRuntime()
    {
      if ( m_finalize ) {
        try { finalize_runtime(); } catch ( ... ) { }
      }
    }
    ScopedRuntime( ScopedRuntime const& ) = delete;
    ScopedRuntime& operator=( ScopedRuntime const& ) = delete;
    ScopedRuntime( ScopedRuntime&& ) = delete;
    ScopedRuntime& operator=( ScopedRuntime&& ) = delete;

  private:
    bool m_finalize;
  };

  namespace detail {
    /** The context, brought up on first use like the reference's implicit runtime. */
    inline dvg_context*
    context( )
    {
      initialize_runtime();
      return runtime_state().ctx;
    }
  }  // namespace detail
}  // namespace diverg

#endif  // DIVERG_B200_RUNTIME_HPP__
