/*
 * gprm_configspace.hpp - drop-in Configspace<ndof> over the C ABI.
 *
 * B200RobotConfigspace<ndof> implements GPUPRM's planner-facing interface
 * Configspace<ndof> (prm/src/lib/prm/configspace.hpp:10-50) with the B200
 * checker, so PRMSolver<ndof> (prm/src/lib/prm/prmsolver.h:74) can be
 * constructed with it in place of RobotConfigspace<ndof>
 * (prm/src/lib/robotspace/robotconfigspace.h:25-176):
 *
 *     #include <prm/configspace.hpp>          // the reference's interface
 *     #include "gprm_configspace.hpp"
 *     B200RobotConfigspace<4> space("../config1", dq, 2 * nbuf);
 *     space.init(rank, size);
 *     PRMSolver<4> prm(&space, distH, distD, maxstorage, blocksize);
 *
 * Include the reference's configspace.hpp first (this header only needs
 * the Configspace<ndof> declaration).  Semantics follow the reference;
 * failures the reference would assert on throw std::runtime_error with
 * the library's message.
 */
#ifndef GPRM_CONFIGSPACE_HPP
#define GPRM_CONFIGSPACE_HPP

#include <stdexcept>
#include <string>

#include "gprm_b200.h"

template <int ndof>
class B200RobotConfigspace : public Configspace<ndof>
{
public:
    /* RobotConfigspace(path, dq, nbuf) (robotconfigspace.cpp:84-98) */
    B200RobotConfigspace(const std::string& path, float dq, int nbuf) : h_(nullptr)
    {
        throw_on_error(gprm_create_from_dir(path.c_str(), ndof, dq, nbuf, &h_), nullptr);
    }
    /* RobotConfigspace(robot, polys, ...) (robotconfigspace.cpp:75-82) */
    B200RobotConfigspace(const gprm_scene_desc& desc, float dq, int nbuf) : h_(nullptr)
    {
        throw_on_error(gprm_create(&desc, dq, nbuf, &h_), nullptr);
    }
    ~B200RobotConfigspace() { gprm_destroy(h_); }
    B200RobotConfigspace(const B200RobotConfigspace&) = delete;
    B200RobotConfigspace& operator=(const B200RobotConfigspace&) = delete;

    int init(const int rank = 0, const int size = 1) { return throw_on_error(gprm_init(h_, rank, size)); }

    int indicator(const float* q, int* res, const int N, const int offset)
    {
        return throw_on_error(gprm_indicator_batch(h_, q, res, N, offset));
    }
    int indicator(const float* q)
    {
        int code = 0;
        throw_on_error(gprm_indicator(h_, q, &code));
        return code;
    }
    int indicator2(const float* qs, const float* qe, int* res, const int N, const int offset)
    {
        return throw_on_error(gprm_indicator2(h_, qs, qe, res, N, offset));
    }
    int indicator2_async(const float* qs, const float* qe, int* res, const int N, const int offset, int& request)
    {
        return throw_on_error(gprm_indicator2_async(h_, qs, qe, res, N, offset, &request));
    }
    int indicator2_async_wait(int request) { return throw_on_error(gprm_indicator2_wait(h_, request)); }
    /* the compressed form is declared but unimplemented in the reference
       too (robotconfigspace.cpp:765-772) */
    /* the compressed edge check (unimplemented in the reference's robot
       space; the meaning of its array space) */
    int indicator2(const float* qs, const int M, const float* qe, int* res, const int* posqe, const int* numqe,
                   const int offset)
    {
        return throw_on_error(gprm_indicator2_compressed(h_, qs, M, qe, res, posqe, numqe, offset));
    }
    int check_boundaries(const float* q, int* res, const int N, const int offset)
    {
        return throw_on_error(gprm_check_boundaries(h_, q, res, N, offset));
    }
    int check_boundaries(const float* q)
    {
        int out = 0;
        throw_on_error(gprm_check_boundaries1(h_, q, &out));
        return out;
    }
    float min(int i) { return gprm_min(h_, i); }
    float max(int i) { return gprm_max(h_, i); }
    float deltaq() { return gprm_deltaq(h_); }
    int dim() { return gprm_dim(h_); }

    gprm_space* handle() { return h_; }

private:
    int throw_on_error(int rc) { return throw_on_error(rc, h_); }
    static int throw_on_error(int rc, gprm_space* h)
    {
        if (rc != GPRM_OK) throw std::runtime_error(std::string("gprm: ") + gprm_last_error(h));
        return 0;
    }
    gprm_space* h_;
};

#endif /* GPRM_CONFIGSPACE_HPP */
