// C shim over the job server's admission queue (bt-am_b200/csrc/sched.hpp),
// built with g++ for the CPU tests of the admission rule.
#include "../../bt-am_b200/csrc/sched.hpp"

extern "C" {
void *sq_create(unsigned long long budget) { return new btam::AdmissionQueue(budget); }
void sq_destroy(void *q) { delete static_cast<btam::AdmissionQueue *>(q); }
void sq_push(void *q, long long id, unsigned long long bytes) {
  static_cast<btam::AdmissionQueue *>(q)->push(id, bytes);
}
long long sq_admit(void *q) { return static_cast<btam::AdmissionQueue *>(q)->admit(); }
void sq_release(void *q, unsigned long long bytes) {
  static_cast<btam::AdmissionQueue *>(q)->release(bytes);
}
unsigned long long sq_in_use(void *q) { return static_cast<btam::AdmissionQueue *>(q)->in_use(); }
int sq_fits_ever(void *q, unsigned long long bytes) {
  return static_cast<btam::AdmissionQueue *>(q)->fits_ever(bytes);
}
}
