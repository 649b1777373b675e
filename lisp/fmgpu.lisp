;;; -*- mode: lisp; -*-
;;;
;;; fmgpu.lisp -- Femlisp binding of libfmgpu.so (the B200 multigrid solve
;;; path) and the drop-in iteration classes built on it.
;;;
;;; The binding uses Femlisp's own foreign-function layer
;;; (src/basic/port.lisp:360-547) the way src/alien/superlu.lisp:57-75 does:
;;; fl.port:def-function declares each C function, fl.port:foreign-call pins
;;; the Lisp arrays and passes their vector-sap.  Argument types are those
;;; convert-type hands to SBCL's define-alien-routine: :int and :double, which
;;; it maps, and SB-ALIEN type names (long, unsigned-long), which it passes
;;; through.  Opaque handles are integers (sb-alien:unsigned-long, the width
;;; of a pointer); a handle returned through a T** out-parameter lands in a
;;; one-element (unsigned-byte 64) vector.  C strings are NUL-terminated octet
;;; vectors, and the two configuration structs are octet vectors laid out as
;;; the C structs (x86-64), filled with sb-sys:sap-ref-32/-double.
;;;
;;; Drop-in classes (make-iterator, linit.lisp:48-67; solve, solve.lisp:46-71):
;;;   <gpu-geometric-cs>   a <geometric-cs> whose iterator runs one cycle on the
;;;                        GPU (fmg_vcycle); the hierarchy is Femlisp's own
;;;                        multilevel-decomposition (geomg.lisp:109-142),
;;;                        uploaded level by level (fmg_set_matrix)
;;;   <gpu-cg>             a <cg> whose iterator runs one CG step per iterate
;;;                        on the GPU (fmg_cg_start / fmg_cg_step), preconditioned
;;;                        by a <gpu-geometric-cs>
;;;   <gpu-linear-solver>  a <linear-solver> whose solve runs the whole loop on
;;;                        the GPU (fmg_solve) and writes :solution, :status,
;;;                        :step, :defnorm, :reduction and the report back
;;; The iterators exchange their vectors with the host on every call, as the
;;; iterator protocol requires (the solver loop reads the residual on the
;;; host); <gpu-linear-solver> exchanges them once per solve.
;;;
;;; Requires SBCL (sb-sys) and a uniformly refined hierarchical mesh of an
;;; n-cube with Lagrange Q1/Q2 (scalar, or vector-valued with node blocks).
;;; Load with (fl.port:load-foreign-library "libfmgpu.so") after adding the
;;; library path to fl.start's foreign-library configuration
;;; (src/config/femlisp-config.lisp:65-93).

(defpackage "FL.FMGPU"
  (:use "COMMON-LISP")
  (:export "<GPU-GEOMETRIC-CS>" "<GPU-CG>" "<GPU-LINEAR-SOLVER>" "GPU-CONTEXT"
           "UPLOAD-ALGEBRAIC-HIERARCHY" "GPU-SOLVE-MIXED")
  (:documentation "The B200 multigrid solve path behind Femlisp's iteration
interface."))

(in-package "FL.FMGPU")

;;;; constants of include/fmgpu.h

(defconstant +fmg-ok+ 0)
(defconstant +fmg-jacobi+ 0)
(defconstant +fmg-sor+ 1)
(defconstant +fmg-ssc+ 2)
(defconstant +fmg-psc+ 3)
(defconstant +fmg-method-mg+ 0)
(defconstant +fmg-method-cg-mg+ 1)
(defconstant +fmg-multiplicative+ 0)
(defconstant +fmg-additive+ 1)
(defconstant +fmg-csr+ 0)
(defconstant +fmg-ccs+ 1)

;;;; foreign functions

(fl.port:def-function ("fmg_init" fmg-init)
    ((device :int) (ctx (* sb-alien:unsigned-long)))
  :returning :int)

(fl.port:def-function ("fmg_finalize" fmg-finalize)
    ((ctx sb-alien:unsigned-long))
  :returning :int)

(fl.port:def-function ("fmg_last_error" fmg-last-error)
    ((ctx sb-alien:unsigned-long) (buf (* :char)) (len :int))
  :returning :int)

(fl.port:def-function ("fmg_grid_create" fmg-grid-create)
    ((ctx sb-alien:unsigned-long) (dim :int) (order :int) (ncomp :int) (n0 :int)
     (top-level :int) (base-level :int) (dirichlet-mask :int)
     (grid (* sb-alien:unsigned-long)))
  :returning :int)

(fl.port:def-function ("fmg_grid_create_algebraic" fmg-grid-create-algebraic)
    ((ctx sb-alien:unsigned-long) (nlevels :int) (sizes (* sb-alien:long))
     (grid (* sb-alien:unsigned-long)))
  :returning :int)

(fl.port:def-function ("fmg_grid_destroy" fmg-grid-destroy)
    ((grid sb-alien:unsigned-long))
  :returning :int)

(fl.port:def-function ("fmg_set_matrix" fmg-set-matrix)
    ((grid sb-alien:unsigned-long) (level :int) (layout :int) (starts (* :int))
     (indices (* :int)) (vals (* :double)) (n sb-alien:long))
  :returning :int)

(fl.port:def-function ("fmg_set_interpolation" fmg-set-interpolation)
    ((grid sb-alien:unsigned-long) (fine-level :int) (layout :int) (starts (* :int))
     (indices (* :int)) (vals (* :double)) (nfine sb-alien:long) (ncoarse sb-alien:long))
  :returning :int)

(fl.port:def-function ("fmg_set_rhs" fmg-set-rhs)
    ((grid sb-alien:unsigned-long) (vals (* :double)) (n sb-alien:long))
  :returning :int)

(fl.port:def-function ("fmg_vec_create" fmg-vec-create)
    ((grid sb-alien:unsigned-long) (level :int) (vec (* sb-alien:unsigned-long)))
  :returning :int)

(fl.port:def-function ("fmg_vec_destroy" fmg-vec-destroy)
    ((vec sb-alien:unsigned-long))
  :returning :int)

(fl.port:def-function ("fmg_vec_set" fmg-vec-set)
    ((vec sb-alien:unsigned-long) (host (* :double)) (n sb-alien:long))
  :returning :int)

(fl.port:def-function ("fmg_vec_get" fmg-vec-get)
    ((vec sb-alien:unsigned-long) (host (* :double)) (n sb-alien:long))
  :returning :int)

;;; one application of the <geometric-cs> iterator (b and r may be the same
;;; vector: the alias inside <cg>, krylow.lisp:120)
(fl.port:def-function ("fmg_vcycle" fmg-vcycle)
    ((grid sb-alien:unsigned-long) (cfg (* :char)) (x sb-alien:unsigned-long)
     (b sb-alien:unsigned-long) (r sb-alien:unsigned-long))
  :returning :int)

;;; the <linear-solver> loop on the device
(fl.port:def-function ("fmg_solve" fmg-solve)
    ((grid sb-alien:unsigned-long) (cfg (* :char)) (x sb-alien:unsigned-long)
     (hist (* :double)) (hist-len :int) (nsteps (* :int)) (status (* :int)))
  :returning :int)

;;; the <cg> iterator one call at a time: initialize and iterate
(fl.port:def-function ("fmg_cg_start" fmg-cg-start)
    ((grid sb-alien:unsigned-long) (cfg (* :char)) (r sb-alien:unsigned-long))
  :returning :int)

(fl.port:def-function ("fmg_cg_step" fmg-cg-step)
    ((grid sb-alien:unsigned-long) (x sb-alien:unsigned-long) (r sb-alien:unsigned-long)
     (defnorm (* :double)))
  :returning :int)

;;; the mixed-precision solve and the learned damping
(fl.port:def-function ("fmg_solve_mixed" fmg-solve-mixed)
    ((grid sb-alien:unsigned-long) (cfg (* :char)) (mcfg (* :char)) (x sb-alien:unsigned-long)
     (hist (* :double)) (hist-len :int) (nouter (* :int)) (ninner (* :int)) (status (* :int)))
  :returning :int)

(fl.port:def-function ("fmg_net_load" fmg-net-load)
    ((ctx sb-alien:unsigned-long) (path (* :char)) (out (* sb-alien:unsigned-long)))
  :returning :int)

(fl.port:def-function ("fmg_net_destroy" fmg-net-destroy)
    ((net sb-alien:unsigned-long))
  :returning :int)

(fl.port:def-function ("fmg_net_apply" fmg-net-apply)
    ((net sb-alien:unsigned-long) (grid sb-alien:unsigned-long))
  :returning :int)

(fl.port:def-function ("fmg_learned_judge_mixed" fmg-learned-judge-mixed)
    ((grid sb-alien:unsigned-long) (cfg (* :char)) (mcfg (* :char)) (rho-plain (* :double))
     (rho-learned (* :double)) (accepted (* :int)))
  :returning :int)

;;;; helpers

(defvar *gpu-context* nil
  "The library context (an integer handle) of this Lisp image, made on first use.")

(defun %u64-cell ()
  (make-array 1 :element-type '(unsigned-byte 64) :initial-element 0))

(defun %last-error ()
  (let ((buf (make-array 512 :element-type '(unsigned-byte 8) :initial-element 0)))
    (when *gpu-context*
      (fl.port:foreign-call #'fmg-last-error *gpu-context* buf (length buf)))
    (map 'string #'code-char (subseq buf 0 (or (position 0 buf) (length buf))))))

(defun check (status what)
  "Femlisp's own alien calls return the status (alien.lisp:151-167); here a
non-zero status is an error carrying the library's message."
  (unless (= status +fmg-ok+)
    (error "libfmgpu: ~A failed with status ~D: ~A" what status (%last-error))))

(defun gpu-context ()
  (or *gpu-context*
      (let ((cell (%u64-cell)))
        (check (fl.port:foreign-call #'fmg-init 0 cell) "fmg_init")
        (setq *gpu-context* (aref cell 0)))))

(defun %c-string (string)
  "STRING as a NUL-terminated octet vector (a const char* for foreign-call)."
  (let ((v (make-array (1+ (length string)) :element-type '(unsigned-byte 8) :initial-element 0)))
    (loop for ch across string for i from 0 do (setf (aref v i) (char-code ch)))
    v))

(defun %struct (size &rest fields)
  "An octet vector of SIZE bytes laid out as a C struct; FIELDS are
(offset :int value) or (offset :double value)."
  (let ((v (make-array size :element-type '(unsigned-byte 8) :initial-element 0)))
    #+sbcl
    (sb-sys:with-pinned-objects (v)
      (let ((sap (sb-sys:vector-sap v)))
        (loop for (off type value) in fields do
          (ecase type
            (:int (setf (sb-sys:sap-ref-32 sap off) (ldb (byte 32 0) value)))
            (:double (setf (sb-sys:sap-ref-double sap off) (coerce value 'double-float)))))))
    #-sbcl (error "fl.fmgpu: the configuration structs are laid out with SBCL's sb-sys")
    v))

(defun %cfg-bytes (&key method smoother damp (pre 1) (post 1) (gamma 1) (compat-alias 0)
                        (coarse-damp 1d0) (rtol 0d0) (atol 0d0) (maxsteps 1)
                        (combination +fmg-multiplicative+) (fmg 0))
  "fmg_solve_cfg (72 bytes on x86-64)."
  (%struct 72 `(0 :int ,method) `(4 :int ,smoother) `(8 :double ,damp)
           `(16 :int ,pre) `(20 :int ,post) `(24 :int ,gamma) `(28 :int ,compat-alias)
           `(32 :double ,coarse-damp) `(40 :double ,rtol) `(48 :double ,atol)
           `(56 :int ,maxsteps) `(60 :int ,combination) `(64 :int ,fmg)))

(defun %mixed-cfg-bytes (&key (max-outer 20) (matrix-free t) (judge 0))
  "fmg_mixed_cfg (24 bytes on x86-64)."
  (%struct 24 '(0 :double 0d0) '(8 :int 0) `(12 :int ,max-outer) `(16 :int ,(if matrix-free 1 0))
           `(20 :int ,judge)))

;;;; the key <-> index numbering of a level

(defun lexicographic-keys (matrix)
  "The row keys of MATRIX in the library's node order: by the midpoint of the
key's cell, last coordinate slowest.  Midpoints of a uniformly refined
n-cube are dyadic, so the comparisons are exact.  The order is the numbering
that sparse-matrix->ccs builds from the keys it is given
(sparselu.lisp:226-263)."
  (let ((keys (coerce (fl.matlisp:row-keys matrix) 'vector)))
    (flet ((mid (key) (fl.mesh:midpoint (fl.mesh:representative key))))
      (sort keys (lambda (a b)
                   (let ((pa (mid a)) (pb (mid b)))
                     (loop for k from (1- (length pa)) downto 0
                           when (< (aref pa k) (aref pb k)) return t
                           when (> (aref pa k) (aref pb k)) return nil
                           finally (return nil))))))))

(defun %block-size (matrix key)
  "Components per node: the number of rows of the diagonal block."
  (fl.matlisp:nrows (fl.matlisp:mref matrix key key)))

;;;; device hierarchies of a matrix

(defstruct (gpu-hierarchy (:conc-name gh-))
  grid keys nc n order x b r)

(defvar *hierarchies* (make-hash-table :test 'eq #+sbcl :weakness #+sbcl :key)
  "Device hierarchies by matrix, made once per matrix.")

(defun %vec (grid level)
  (let ((cell (%u64-cell)))
    (check (fl.port:foreign-call #'fmg-vec-create grid level cell) "fmg_vec_create")
    (aref cell 0)))

(defun %to-device (h svec dvec)
  "Copies the <sparse-vector> SVEC (blocks of nc x 1 per key) into the device
vector DVEC in the hierarchy's node order."
  (let* ((nc (gh-nc h)) (keys (gh-keys h))
         (host (make-array (gh-n h) :element-type 'double-float :initial-element 0d0)))
    (loop for key across keys for i from 0
          for blk = (fl.matlisp:store (fl.matlisp:vref svec key)) do
            (dotimes (k nc) (setf (aref host (+ (* nc i) k)) (aref blk k))))
    (check (fl.port:foreign-call #'fmg-vec-set dvec host (length host)) "fmg_vec_set")
    host))

(defun %from-device (h dvec svec)
  "Copies the device vector DVEC back into the blocks of SVEC."
  (let* ((nc (gh-nc h)) (keys (gh-keys h))
         (host (make-array (gh-n h) :element-type 'double-float :initial-element 0d0)))
    (check (fl.port:foreign-call #'fmg-vec-get dvec host (length host)) "fmg_vec_get")
    (loop for key across keys for i from 0
          for blk = (fl.matlisp:store (fl.matlisp:vref svec key)) do
            (dotimes (k nc) (setf (aref blk k) (aref host (+ (* nc i) k)))))
    svec))

(defun %upload-level (grid level matrix keys)
  "fmg_set_matrix with the compressed columns of sparse-matrix->ccs in the
key order KEYS."
  (let* ((ccs (fl.matlisp:sparse-matrix->ccs matrix :keys keys))
         (pattern (fl.matlisp:pattern ccs)))
    (check (fl.port:foreign-call #'fmg-set-matrix grid level +fmg-ccs+
                                 (slot-value pattern 'fl.matlisp::starts)
                                 (slot-value pattern 'fl.matlisp::indices)
                                 (fl.matlisp:store ccs)
                                 (* (%block-size matrix (aref keys 0)) (length keys)))
           "fmg_set_matrix")))

;;;; <gpu-geometric-cs>

(defclass <gpu-geometric-cs> (fl.geomg:<geometric-cs>)
  ((dirichlet-mask :initarg :dirichlet-mask :initform nil
                   :documentation "Faces carrying essential constraints, bit 2k the
lower and 2k+1 the upper face of direction k; NIL: all faces (the default of
cdr-model-problem)."))
  (:documentation "A <geometric-cs> whose cycles run on the GPU.  The level
matrices are Femlisp's own (multilevel-decomposition of <geometric-mg>,
geomg.lisp:109-142), handed to the device once per matrix; the smoother
(<jacobi>, <sor>, geometric-ssc, geometric-psc), the steps, gamma, the
combination, :fmg and the <lu> coarse-grid iteration are this object's."))

(defun %smoother-code (smoother order)
  "FMG_* code and :damp/:omega of SMOOTHER: a <jacobi>, <sor> or <gauss-seidel>
iteration, a geometric-ssc or geometric-psc, or NIL for select-smoother's
default (geomg.lisp:48-60): Gauss-Seidel for order 1, SSC above."
  (cond ((null smoother)
         (if (eql order 1) (values +fmg-sor+ 1d0) (values +fmg-ssc+ 1d0)))
        ((typep smoother 'fl.iteration:<jacobi>)
         (values +fmg-jacobi+ (slot-value smoother 'fl.iteration::damp)))
        ((typep smoother 'fl.iteration:<sor>)
         (values +fmg-sor+ (slot-value smoother 'fl.iteration::omega)))
        ((typep smoother 'fl.iteration::<psc>)
         (values +fmg-psc+ (slot-value smoother 'fl.iteration::damp)))
        ((typep smoother 'fl.iteration::<ssc>)
         (values +fmg-ssc+ (slot-value smoother 'fl.iteration::omega)))
        (t (error "fl.fmgpu: no GPU form of the smoother ~S" smoother))))

(defun %mg-cfg (mgit method order &key (rtol 0d0) (atol 0d0) (maxsteps 1) (compat-alias 0))
  "fmg_solve_cfg from the initargs of the <gpu-geometric-cs> MGIT (ORDER: the
discretization order, for the default smoother)."
  (multiple-value-bind (code damp)
      (%smoother-code (and (slot-boundp mgit 'fl.multigrid::pre-smoother)
                           (slot-value mgit 'fl.multigrid::pre-smoother))
                      order)
    (let ((cgi (fl.multigrid:coarse-grid-iteration mgit)))
      (%cfg-bytes :method method :smoother code :damp (coerce damp 'double-float)
                  :pre (fl.multigrid:pre-steps mgit) :post (fl.multigrid:post-steps mgit)
                  :gamma (slot-value mgit 'fl.multigrid::gamma)
                  :compat-alias compat-alias
                  :coarse-damp (if (typep cgi 'fl.iteration:<lu>) (slot-value cgi 'fl.iteration::damp) 1d0)
                  :rtol rtol :atol atol :maxsteps maxsteps
                  :combination (if (eq (slot-value mgit 'fl.multigrid::combination) :additive)
                                   +fmg-additive+ +fmg-multiplicative+)
                  :fmg (if (fl.multigrid:fmg mgit) 1 0)))))

(defgeneric gpu-hierarchy (mgit matrix)
  (:documentation "The device hierarchy of MATRIX for the GPU multigrid
iteration MGIT and three top-level device vectors, made once per matrix.
The hierarchy lives as long as the matrix (a weak table on SBCL)."))

(defmethod gpu-hierarchy ((mgit <gpu-geometric-cs>) matrix)
  "A structured grid of the same levels, every level matrix from Femlisp's
multilevel decomposition in the library's lexicographic node order."
  (or (gethash matrix *hierarchies*)
      (let* ((as (fl.discretization:ansatz-space matrix))
             (h-mesh (fl.discretization:hierarchical-mesh as))
             (dim (fl.mesh:dimension h-mesh))
             (top (fl.mesh:top-level h-mesh))
             (base (fl.multigrid:base-level mgit))
             (order (fl.discretization:discretization-order as))
             (n0 (round (expt (length (fl.mesh:cells-on-level h-mesh 0)) (/ 1 dim))))
             (mask (or (slot-value mgit 'dirichlet-mask) (1- (expt 2 (* 2 dim)))))
             (mg-data (fl.multigrid:multilevel-decomposition mgit matrix))
             (a-vec (fl.utilities:getbb mg-data :a-vec))
             (keys (lexicographic-keys matrix))
             (nc (%block-size matrix (aref keys 0)))
             (cell (%u64-cell)))
        (check (fl.port:foreign-call #'fmg-grid-create (gpu-context) dim order nc n0 top base mask cell)
               "fmg_grid_create")
        (let ((grid (aref cell 0)))
          (loop for level from base upto top
                for l-mat = (aref a-vec level) do
                  (%upload-level grid level l-mat (if (= level top) keys (lexicographic-keys l-mat))))
          (setf (gethash matrix *hierarchies*)
                (make-gpu-hierarchy :grid grid :keys keys :nc nc :n (* nc (length keys)) :order order
                                    :x (%vec grid top) :b (%vec grid top) :r (%vec grid top)))))))

(defmethod fl.iteration:make-iterator ((mgit <gpu-geometric-cs>) (matrix fl.matlisp:<sparse-matrix>))
  "The <mg-iteration> iterator (multigrid.lisp:303-393) with the cycle on the
GPU: the top-level solution, rhs and residual are the given vectors, updated
in place; the same vector as rhs and residual is the alias of <cg>'s
preconditioner call."
  (let* ((h (gpu-hierarchy mgit matrix))
         (cfg (%mg-cfg mgit +fmg-method-mg+ (gh-order h))))
    (make-instance
     'fl.iteration:<iterator>
     :matrix matrix
     :residual-before t
     :initialize nil
     :iterate (lambda (x b r)
                (let ((alias (eq b r)))
                  (%to-device h x (gh-x h))
                  (%to-device h b (gh-b h))
                  (unless alias (%to-device h r (gh-r h)))
                  (check (fl.port:foreign-call #'fmg-vcycle (gh-grid h) cfg (gh-x h) (gh-b h)
                                               (if alias (gh-b h) (gh-r h)))
                         "fmg_vcycle")
                  (%from-device h (gh-x h) x)
                  (%from-device h (gh-b h) b)
                  (unless alias (%from-device h (gh-r h) r))
                  x))
     :residual-after nil)))

;;;; <gpu-local-mg>

(defclass <gpu-local-mg> (<gpu-geometric-cs> fl.geomg::<local-mg>)
  ()
  (:documentation "A <local-mg> (geomg.lisp:161-168) whose cycles run on the
GPU over an algebraic device hierarchy, so that the mesh may be refined
locally: the level matrices and the constrained interpolations of Femlisp's
multilevel decomposition (geomg.lisp:109-142; hanging-node and essential
constraints eliminated on the host, constraints.lisp:58-151,323-411) handed
over as compressed columns in each level's own key order.  Scalar problems;
smoothers <jacobi>, <sor> and <gauss-seidel> (the rows ordered by a greedy
colouring of each level's matrix graph) and geometric-ssc (one-unknown
blocks).  make-iterator, <gpu-cg> and <gpu-linear-solver> take it like a
<gpu-geometric-cs>."))

(defun %upload-interpolation (grid level imat row-keys col-keys)
  "fmg_set_interpolation with the compressed columns of IMAT (rows: the keys
of LEVEL, columns: the keys of the level below)."
  (let* ((ccs (fl.matlisp:sparse-matrix->ccs imat :row-keys row-keys :col-keys col-keys))
         (pattern (fl.matlisp:pattern ccs)))
    (check (fl.port:foreign-call #'fmg-set-interpolation grid level +fmg-ccs+
                                 (slot-value pattern 'fl.matlisp::starts)
                                 (slot-value pattern 'fl.matlisp::indices)
                                 (fl.matlisp:store ccs) (length row-keys) (length col-keys))
           "fmg_set_interpolation")))

(defmethod gpu-hierarchy ((mgit <gpu-local-mg>) matrix)
  "An algebraic grid of the levels base .. top of the multilevel
decomposition renumbered from 0: the a-vec matrices, and the i-vec
interpolation from each level to the next (constrained-interpolation-matrix,
constraints.lisp:58-72)."
  (or (gethash matrix *hierarchies*)
      (let* ((as (fl.discretization:ansatz-space matrix))
             (top (fl.mesh:top-level (fl.discretization:hierarchical-mesh as)))
             (base (fl.multigrid:base-level mgit))
             (mg-data (fl.multigrid:multilevel-decomposition mgit matrix))
             (a-vec (fl.utilities:getbb mg-data :a-vec))
             (i-vec (fl.utilities:getbb mg-data :i-vec))
             (keys (loop for level from base upto top
                         collect (coerce (fl.matlisp:row-keys (aref a-vec level)) 'vector)))
             (sizes (map '(vector (signed-byte 64)) #'length keys))
             (ltop (- top base))
             (cell (%u64-cell)))
        (unless (= 1 (%block-size matrix (aref (nth ltop keys) 0)))
          (error "fl.fmgpu: <gpu-local-mg> takes scalar problems"))
        (check (fl.port:foreign-call #'fmg-grid-create-algebraic (gpu-context) (length sizes) sizes cell)
               "fmg_grid_create_algebraic")
        (let ((grid (aref cell 0)))
          (loop for k in keys for level from 0 do
            (%upload-level grid level (aref a-vec (+ base level)) k))
          (loop for level from 1 upto ltop do
            (%upload-interpolation grid level (aref i-vec (+ base level -1)) (nth level keys)
                                   (nth (1- level) keys)))
          (setf (gethash matrix *hierarchies*)
                (make-gpu-hierarchy :grid grid :keys (nth ltop keys) :nc 1 :n (length (nth ltop keys))
                                    :order (fl.discretization:discretization-order as)
                                    :x (%vec grid ltop) :b (%vec grid ltop) :r (%vec grid ltop)))))))

;;;; <gpu-cg>

(defclass <gpu-cg> (fl.iteration:<cg>)
  ()
  (:documentation "A <cg> whose steps run on the GPU; its preconditioner
must be a <gpu-geometric-cs>."))

(defmethod fl.iteration:make-iterator ((cg <gpu-cg>) (matrix fl.matlisp:<sparse-matrix>))
  "The <cg> iterator (krylow.lisp:72-132): initialize restarts from the
residual (fmg_cg_start), each iterate is one CG step (fmg_cg_step) after
which the solution and the residual are back in the given vectors."
  (let ((pre (slot-value cg 'fl.iteration::preconditioner)))
    (unless (typep pre '<gpu-geometric-cs>)
      (error "fl.fmgpu: <gpu-cg> needs a <gpu-geometric-cs> preconditioner, not ~S" pre))
    (let* ((h (gpu-hierarchy pre matrix))
           (cfg (%mg-cfg pre +fmg-method-cg-mg+ (gh-order h)))
           (defnorm (make-array 1 :element-type 'double-float :initial-element 0d0)))
      (make-instance
       'fl.iteration:<iterator>
       :matrix matrix
       :residual-before t
       :initialize (lambda (x b r)
                     (declare (ignore b))
                     (%to-device h x (gh-x h))
                     (%to-device h r (gh-r h))
                     (check (fl.port:foreign-call #'fmg-cg-start (gh-grid h) cfg (gh-r h)) "fmg_cg_start"))
       :iterate (lambda (x b r)
                  (declare (ignore b))
                  (check (fl.port:foreign-call #'fmg-cg-step (gh-grid h) (gh-x h) (gh-r h) defnorm)
                         "fmg_cg_step")
                  (%from-device h (gh-x h) x)
                  (%from-device h (gh-r h) r)
                  (list :residual-after t))
       :residual-after t))))

;;;; <gpu-linear-solver>

(defclass <gpu-linear-solver> (fl.iteration:<linear-solver>)
  ()
  (:documentation "A <linear-solver> whose whole loop runs on the GPU.  Its
:iteration is a <gpu-cg> (preconditioned by a <gpu-geometric-cs>) or a
<gpu-geometric-cs>; its success and failure forms may combine (< :reduction
r), (< :defnorm d) and (> :step n) with OR."))

(defun %termination (success failure)
  "rtol, atol and the step limit of the success/failure forms."
  (let ((rtol 0d0) (atol 0d0) (maxsteps nil))
    (labels ((walk (form)
               (when (consp form)
                 (case (car form)
                   (or (mapc #'walk (cdr form)))
                   (< (case (second form)
                        (:reduction (setq rtol (coerce (third form) 'double-float)))
                        (:defnorm (setq atol (coerce (third form) 'double-float)))))
                   (> (when (eq (second form) :step) (setq maxsteps (third form))))
                   (>= (when (eq (second form) :step) (setq maxsteps (1- (third form)))))))))
      (walk success)
      (walk failure))
    (values rtol atol (or maxsteps 100))))

(defmethod fl.iteration:solve ((solver <gpu-linear-solver>) &optional blackboard)
  "Solves the linear system on BLACKBOARD (:matrix and :rhs, or a :problem
carrying them; :solution as the initial guess if present) on the GPU and
returns the blackboard with :solution, :status, :step, :defnorm,
:initial-defnorm, :reduction and the convergence rate in :report."
  (fl.utilities:with-items (&key problem matrix rhs solution status step defnorm initial-defnorm reduction
                                 report)
      blackboard
    (let* ((a (or matrix (fl.problem:matrix problem)))
           (b (or rhs (fl.problem:rhs problem)))
           (it (slot-value solver 'fl.iteration::iteration))
           (cgp (typep it '<gpu-cg>))
           (mgit (if cgp (slot-value it 'fl.iteration::preconditioner) it)))
      (unless (typep mgit '<gpu-geometric-cs>)
        (error "fl.fmgpu: <gpu-linear-solver> runs a <gpu-cg> or a <gpu-geometric-cs>, not ~S" it))
      (multiple-value-bind (rtol atol maxsteps)
          (%termination (slot-value solver 'fl.iteration:success-if)
                        (slot-value solver 'fl.iteration:failure-if))
        (let* ((h (gpu-hierarchy mgit a))
               (cfg (%mg-cfg mgit (if cgp +fmg-method-cg-mg+ +fmg-method-mg+) (gh-order h)
                             :rtol rtol :atol atol :maxsteps maxsteps))
               (hist (make-array (+ maxsteps 2) :element-type 'double-float :initial-element 0d0))
               (nsteps (make-array 1 :element-type '(signed-byte 32) :initial-element 0))
               (st (make-array 1 :element-type '(signed-byte 32) :initial-element 0)))
          (check (fl.port:foreign-call #'fmg-set-rhs (gh-grid h) (%to-device h b (gh-b h)) (gh-n h))
                 "fmg_set_rhs")
          (unless solution
            (setq solution (fl.matlisp:make-domain-vector-for a)))
          (%to-device h solution (gh-x h))
          (check (fl.port:foreign-call #'fmg-solve (gh-grid h) cfg (gh-x h) hist (length hist) nsteps st)
                 "fmg_solve")
          (%from-device h (gh-x h) solution)
          (let ((k (aref nsteps 0)))
            (setq status (if (zerop (aref st 0)) :success :failure)
                  step k
                  initial-defnorm (aref hist 0)
                  defnorm (aref hist k)
                  reduction (if (zerop (aref hist 0)) 0d0 (/ (aref hist k) (aref hist 0))))
            (unless report (setq report (fl.utilities:blackboard)))
            (setf (fl.utilities:getbb report :convergence-rate)
                  (if (plusp k) (expt reduction (/ 1d0 k)) :undefined))
            (setf (fl.utilities:getbb report :defnorm-history) (subseq hist 0 (1+ k)))))))
    blackboard))

;;;; hierarchies on unstructured or adaptively refined meshes

(defun upload-algebraic-hierarchy (matrices interpolations rhs)
  "MATRICES: the level matrices of a multilevel decomposition, coarsest first
(<sparse-matrix>, constraints eliminated; multilevel-decomposition,
geomg.lisp:109-142); INTERPOLATIONS: the constrained interpolation into each
level above the coarsest (constrained-interpolation-matrix,
constraints.lisp:58-72), coarsest first; RHS: the top-level right-hand side as
a double vector in the top level's key order.  Returns the grid handle."
  (let* ((keys (mapcar (lambda (m) (coerce (fl.matlisp:row-keys m) 'vector)) matrices))
         (sizes (map '(vector (signed-byte 64)) #'length keys))
         (cell (%u64-cell)))
    (check (fl.port:foreign-call #'fmg-grid-create-algebraic (gpu-context) (length sizes) sizes cell)
           "fmg_grid_create_algebraic")
    (let ((grid (aref cell 0)))
      (loop for m in matrices for k in keys for level from 0 do
        (let* ((ccs (fl.matlisp:sparse-matrix->ccs m :keys k))
               (pattern (fl.matlisp:pattern ccs)))
          (check (fl.port:foreign-call #'fmg-set-matrix grid level +fmg-ccs+
                                       (slot-value pattern 'fl.matlisp::starts)
                                       (slot-value pattern 'fl.matlisp::indices)
                                       (fl.matlisp:store ccs) (length k))
                 "fmg_set_matrix")))
      (loop for i in interpolations for level from 1 do
        (%upload-interpolation grid level i (nth level keys) (nth (1- level) keys)))
      (check (fl.port:foreign-call #'fmg-set-rhs grid rhs (length rhs)) "fmg_set_rhs")
      grid)))

;;;; the mixed-precision solve with the learned damping

(defun gpu-solve-mixed (grid level weights-path &key (damp 0.6d0) (reduction 1d-10) (maxsteps 200))
  "On an assembled GRID whose top level is LEVEL: installs the per-node damping
the network in WEIGHTS-PATH predicts, lets the plain cycle judge it (it stays
only if no worse), and solves with FP64 flexible CG around the FP32/BF16
V(1,1) Jacobi cycle.  Returns the solution vector handle and the :defnorm
history."
  (let* ((ctx (gpu-context))
         (net (%u64-cell))
         (x (%u64-cell))
         (cfg (%cfg-bytes :method +fmg-method-cg-mg+ :smoother +fmg-jacobi+ :damp damp
                          :rtol reduction :maxsteps maxsteps))
         (mcfg (%mixed-cfg-bytes))
         (rho-plain (make-array 1 :element-type 'double-float :initial-element 0d0))
         (rho-learned (make-array 1 :element-type 'double-float :initial-element 0d0))
         (accepted (make-array 1 :element-type '(signed-byte 32) :initial-element 0))
         (hist (make-array (+ maxsteps 24) :element-type 'double-float :initial-element 0d0))
         (nouter (make-array 1 :element-type '(signed-byte 32) :initial-element 0))
         (ninner (make-array 1 :element-type '(signed-byte 32) :initial-element 0))
         (status (make-array 1 :element-type '(signed-byte 32) :initial-element 0)))
    (check (fl.port:foreign-call #'fmg-net-load ctx (%c-string (namestring weights-path)) net) "fmg_net_load")
    (unwind-protect
         (progn
           (check (fl.port:foreign-call #'fmg-net-apply (aref net 0) grid) "fmg_net_apply")
           (check (fl.port:foreign-call #'fmg-learned-judge-mixed grid cfg mcfg rho-plain rho-learned accepted)
                  "fmg_learned_judge_mixed"))
      (fl.port:foreign-call #'fmg-net-destroy (aref net 0)))
    (check (fl.port:foreign-call #'fmg-vec-create grid level x) "fmg_vec_create")
    (check (fl.port:foreign-call #'fmg-solve-mixed grid cfg mcfg (aref x 0) hist (length hist)
                                 nouter ninner status)
           "fmg_solve_mixed")
    (values (aref x 0) (subseq hist 0 (+ (aref nouter 0) (aref ninner 0) 1)))))
