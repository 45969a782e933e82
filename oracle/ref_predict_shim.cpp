// ref_predict_shim.cpp -- plain C entry points around the reference's own compile_trees_cpp / predict_draw_cpp
// (src/predict.cpp:12-73, compiled unmodified against oracle/rcpp_stub/Rcpp.h).  TEST INFRASTRUCTURE ONLY: the
// checker that pins this project's evaluator oracle (and, through it, the device evaluators) to the reference.
#include <cstring>
#include <string>

#include "Rcpp.h"

Rcpp::List compile_trees_cpp(std::string trees, Rcpp::List cutpoints);
Rcpp::NumericVector predict_draw_cpp(Rcpp::List ct, Rcpp::List newdata, int m, double mu);

namespace {
void set_err(char* err, int cap, const char* msg) {
  if (err && cap > 0) {
    std::strncpy(err, msg, static_cast<size_t>(cap - 1));
    err[cap - 1] = 0;
  }
}
}  // namespace

extern "C" {

// compile_trees_cpp on tree text and ncol cutpoint vectors; returns a handle (NULL on error, message in err)
void* refp_compile(const char* text, const double* const* cps, const int* ncut, int ncol, char* err, int errcap) {
  try {
    Rcpp::List cl;
    for (int v = 0; v < ncol; v++)
      cl.items.push_back({"", Rcpp::Value(std::vector<double>(cps[v], cps[v] + ncut[v]))});
    return new Rcpp::List(compile_trees_cpp(std::string(text), cl));
  } catch (const std::exception& e) {
    set_err(err, errcap, e.what());
    return nullptr;
  }
}

// ndpost, ntree, p and the number of nodes of a compiled result
void refp_info(void* h, int* nd, int* m, int* p, int* nnodes) {
  Rcpp::List& ct = *static_cast<Rcpp::List*>(h);
  *nd = Rcpp::as<int>(ct["ndpost"]);
  *m = Rcpp::as<int>(ct["ntree"]);
  *p = Rcpp::as<int>(ct["p"]);
  *nnodes = static_cast<int>(ct["var"].i.size());
}

// copies the node arrays (var, child, cut, theta [nnodes]) and root [ndpost * ntree]
void refp_arrays(void* h, int* var, int* child, double* cut, double* theta, int* root) {
  Rcpp::List& ct = *static_cast<Rcpp::List*>(h);
  const auto& vv = ct["var"].i;
  std::memcpy(var, vv.data(), vv.size() * sizeof(int));
  std::memcpy(child, ct["child"].i.data(), ct["child"].i.size() * sizeof(int));
  std::memcpy(cut, ct["cut"].d.data(), ct["cut"].d.size() * sizeof(double));
  std::memcpy(theta, ct["theta"].d.data(), ct["theta"].d.size() * sizeof(double));
  std::memcpy(root, ct["root"].i.data(), ct["root"].i.size() * sizeof(int));
}

// predict_draw_cpp of draw m (1-based) on ncol columns of n rows; 0 on success, -1 with the reference's message
int refp_predict(void* h, const double* const* cols, int ncol, int n, int m, double mu, double* out, char* err,
                 int errcap) {
  try {
    Rcpp::List nd;
    for (int v = 0; v < ncol; v++) nd.items.push_back({"", Rcpp::Value(std::vector<double>(cols[v], cols[v] + n))});
    Rcpp::NumericVector f = predict_draw_cpp(*static_cast<Rcpp::List*>(h), nd, m, mu);
    std::memcpy(out, f.v.data(), f.v.size() * sizeof(double));
    return 0;
  } catch (const std::exception& e) {
    set_err(err, errcap, e.what());
    return -1;
  }
}

void refp_free(void* h) { delete static_cast<Rcpp::List*>(h); }

}  // extern "C"
