/* generated_bags.hpp -- the C++ the EmptyHeaded query compiler emits for
 * the bags of the reference's test queries, written out by hand.
 *
 * TEST INFRASTRUCTURE ONLY.  The Scala query compiler cannot run in this
 * image (no JVM), so each bag is written statement by statement in the shape
 * EHGenerator.scala emits for the plans pinned by QueryPlannerTest.scala:
 *   - emitHeadParForeach  query_compiler/.../codegen/query/EHGenerator.scala:273-300
 *   - emitBuildCode       EHGenerator.scala:302-354
 *   - emitForeach         EHGenerator.scala:384-397
 *   - annotation code     EHGenerator.scala:399-480
 *   - bag wrapper         EHGenerator.scala:728-838
 * Plans: triangle / 4-clique one bag, order [a,b,(c),(d)]
 * (QueryPlannerTest.scala:78-96); lollipop / barbell two bags with an
 * annotated bag (QueryPlannerTest.scala:199-230, IROptimizerTest.scala:189);
 * the selections of QueryPlannerTest.scala:230-304; and a two-path COUNT,
 * a body no device plan runs.
 *
 * The same source is compiled against two engines: the reference storage
 * engine (oracle/ref_driver.cpp, built from the reference's own sources) and
 * the B200 layer of include/eh/ (tests/cpp/dropin_bags.cpp).  The includer
 * defines MB (the memory-buffer template argument) and includes the engine's
 * Trie.hpp, TrieBuilder.hpp, TrieIterator.hpp and trie/TrieBlock.hpp first.
 */
#ifndef EH_GENERATED_BAGS_HPP
#define EH_GENERATED_BAGS_HPP

#include <sys/stat.h>

#include <string>
#include <vector>
/* ------------------------------------------------- generated-shape bags */

/* TriangleAgg(;z) :- Edge(a,b),Edge(b,c),Edge(a,c),z:long<-[COUNT(*)]. */
static long bag_triangle(Trie<void*, MB>* Trie_Edge_0_1, const std::string& out) {
  Trie<long, MB>* Trie_TriangleAgg_ = new Trie<long, MB>(out, 0, true);
  long result;
  {
    ParTrieBuilder<long, MB> Builders(Trie_TriangleAgg_, 3);
    ParTrieIterator<void*, MB> Iterators_Edge_a_b(Trie_Edge_0_1);
    ParTrieIterator<void*, MB> Iterators_Edge_b_c(Trie_Edge_0_1);
    ParTrieIterator<void*, MB> Iterators_Edge_a_c(Trie_Edge_0_1);
    const size_t count_a = Builders.build_aggregated_set(Iterators_Edge_a_b.head, Iterators_Edge_a_c.head);
    (void)count_a;
    par::reducer<long> annotation_a(0, [&](long a, long b) { return a + b; });
    Builders.par_foreach_aggregate([&](const size_t tid, const uint32_t a_d) {
      TrieBuilder<long, MB>* Builder = Builders.builders.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_a_b = Iterators_Edge_a_b.iterators.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_b_c = Iterators_Edge_b_c.iterators.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_a_c = Iterators_Edge_a_c.iterators.at(tid);
      Iterator_Edge_a_b->get_next_block(0, a_d);
      Iterator_Edge_a_c->get_next_block(0, a_d);
      const size_t count_b =
          Builder->build_aggregated_set(Iterator_Edge_a_b->get_block(1), Iterator_Edge_b_c->get_block(0));
      (void)count_b;
      long annotation_b = (long)0;
      Builder->foreach_aggregate([&](const uint32_t b_d) {
        Iterator_Edge_b_c->get_next_block(0, b_d);
        const size_t count_c =
            Builder->build_aggregated_set(Iterator_Edge_b_c->get_block(1), Iterator_Edge_a_c->get_block(1));
        const long intermediate_c = (long)1 * (count_c * 1);
        annotation_b += intermediate_c;
      });
      annotation_a.update(tid, annotation_b);
    });
    Builders.trie->annotation = annotation_a.evaluate(0);
    result = Builders.trie->annotation;
  }
  delete Trie_TriangleAgg_;
  return result;
}

/* FliqueAgg(;z) :- Edge(a,b),Edge(b,c),Edge(a,c),Edge(a,d),Edge(b,d),Edge(c,d),z:long<-[COUNT(*)]. */
static long bag_clique4(Trie<void*, MB>* Trie_Edge_0_1, const std::string& out) {
  typedef const TrieBlock<hybrid, MB>* TB;
  Trie<long, MB>* Trie_FliqueAgg_ = new Trie<long, MB>(out, 0, true);
  long result;
  {
    ParTrieBuilder<long, MB> Builders(Trie_FliqueAgg_, 4);
    ParTrieIterator<void*, MB> Iterators_Edge_a_b(Trie_Edge_0_1);
    ParTrieIterator<void*, MB> Iterators_Edge_b_c(Trie_Edge_0_1);
    ParTrieIterator<void*, MB> Iterators_Edge_a_c(Trie_Edge_0_1);
    ParTrieIterator<void*, MB> Iterators_Edge_a_d(Trie_Edge_0_1);
    ParTrieIterator<void*, MB> Iterators_Edge_b_d(Trie_Edge_0_1);
    ParTrieIterator<void*, MB> Iterators_Edge_c_d(Trie_Edge_0_1);
    std::vector<TB> a_sets;
    a_sets.push_back(Iterators_Edge_a_b.head);
    a_sets.push_back(Iterators_Edge_a_c.head);
    a_sets.push_back(Iterators_Edge_a_d.head);
    const size_t count_a = Builders.build_aggregated_set(&a_sets);
    (void)count_a;
    par::reducer<long> annotation_a(0, [&](long a, long b) { return a + b; });
    Builders.par_foreach_aggregate([&](const size_t tid, const uint32_t a_d) {
      TrieBuilder<long, MB>* Builder = Builders.builders.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_a_b = Iterators_Edge_a_b.iterators.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_b_c = Iterators_Edge_b_c.iterators.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_a_c = Iterators_Edge_a_c.iterators.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_a_d = Iterators_Edge_a_d.iterators.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_b_d = Iterators_Edge_b_d.iterators.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_c_d = Iterators_Edge_c_d.iterators.at(tid);
      Iterator_Edge_a_b->get_next_block(0, a_d);
      Iterator_Edge_a_c->get_next_block(0, a_d);
      Iterator_Edge_a_d->get_next_block(0, a_d);
      std::vector<TB> b_sets;
      b_sets.push_back(Iterator_Edge_a_b->get_block(1));
      b_sets.push_back(Iterator_Edge_b_c->get_block(0));
      b_sets.push_back(Iterator_Edge_b_d->get_block(0));
      const size_t count_b = Builder->build_aggregated_set(&b_sets);
      (void)count_b;
      long annotation_b = (long)0;
      Builder->foreach_aggregate([&](const uint32_t b_d) {
        Iterator_Edge_b_c->get_next_block(0, b_d);
        Iterator_Edge_b_d->get_next_block(0, b_d);
        std::vector<TB> c_sets;
        c_sets.push_back(Iterator_Edge_b_c->get_block(1));
        c_sets.push_back(Iterator_Edge_a_c->get_block(1));
        c_sets.push_back(Iterator_Edge_c_d->get_block(0));
        const size_t count_c = Builder->build_aggregated_set(&c_sets);
        (void)count_c;
        long annotation_c = (long)0;
        Builder->foreach_aggregate([&](const uint32_t c_d) {
          Iterator_Edge_c_d->get_next_block(0, c_d);
          std::vector<TB> d_sets;
          d_sets.push_back(Iterator_Edge_a_d->get_block(1));
          d_sets.push_back(Iterator_Edge_b_d->get_block(1));
          d_sets.push_back(Iterator_Edge_c_d->get_block(1));
          const size_t count_d = Builder->build_aggregated_set(&d_sets);
          const long intermediate_d = (long)1 * (count_d * 1);
          annotation_c += intermediate_d;
        });
        annotation_b += annotation_c;
      });
      annotation_a.update(tid, annotation_b);
    });
    Builders.trie->annotation = annotation_a.evaluate(0);
    result = Builders.trie->annotation;
  }
  delete Trie_FliqueAgg_;
  return result;
}

/* bag_1_a_b_c(a;z) :- Edge(a,c),Edge(b,c),Edge(a,b),z:long<-[SUM over (b,c) of 1].
 * Materialised 1-level annotated trie (QueryPlannerTest.scala:199-212). */
static Trie<long, MB>* bag_triangle_annot(Trie<void*, MB>* Trie_Edge_0_1, const std::string& out) {
  mkdir(out.c_str(), 0755);
  mkdir((out + "/ram").c_str(), 0755);
  Trie<long, MB>* Trie_bag_1_a_b_c_0 = new Trie<long, MB>(out, 1, true);
  {
    ParTrieBuilder<long, MB> Builders(Trie_bag_1_a_b_c_0, 3);
    ParTrieIterator<void*, MB> Iterators_Edge_a_c(Trie_Edge_0_1);
    ParTrieIterator<void*, MB> Iterators_Edge_b_c(Trie_Edge_0_1);
    ParTrieIterator<void*, MB> Iterators_Edge_a_b(Trie_Edge_0_1);
    const size_t count_a = Builders.build_set(Iterators_Edge_a_c.head, Iterators_Edge_a_b.head);
    Builders.allocate_annotation();
    Builders.par_foreach_builder([&](const size_t tid, const uint32_t a_i, const uint32_t a_d) {
      TrieBuilder<long, MB>* Builder = Builders.builders.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_a_c = Iterators_Edge_a_c.iterators.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_b_c = Iterators_Edge_b_c.iterators.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_a_b = Iterators_Edge_a_b.iterators.at(tid);
      Iterator_Edge_a_c->get_next_block(0, a_d);
      Iterator_Edge_a_b->get_next_block(0, a_d);
      const size_t count_b =
          Builder->build_aggregated_set(Iterator_Edge_b_c->get_block(0), Iterator_Edge_a_b->get_block(1));
      (void)count_b;
      long annotation_b = (long)0;
      Builder->foreach_aggregate([&](const uint32_t b_d) {
        Iterator_Edge_b_c->get_next_block(0, b_d);
        const size_t count_c =
            Builder->build_aggregated_set(Iterator_Edge_a_c->get_block(1), Iterator_Edge_b_c->get_block(1));
        const long intermediate_c = (long)1 * (count_c * 1);
        annotation_b += intermediate_c;
      });
      Builder->set_annotation(annotation_b, a_i, a_d);
    });
    Builders.trie->num_rows = count_a;
  }
  return Trie_bag_1_a_b_c_0;
}

/* LollipopAgg(;z) :- Edge(a,d) ⋈ bag_1(a;z)  (root bag, order [a,d]) */
static long bag_lollipop_root(Trie<void*, MB>* Trie_Edge_0_1, Trie<long, MB>* Trie_bag_1, const std::string& out) {
  Trie<long, MB>* Trie_LollipopAgg_ = new Trie<long, MB>(out, 0, true);
  long result;
  {
    ParTrieBuilder<long, MB> Builders(Trie_LollipopAgg_, 2);
    ParTrieIterator<void*, MB> Iterators_Edge_a_d(Trie_Edge_0_1);
    ParTrieIterator<long, MB> Iterators_bag_1_a(Trie_bag_1);
    const size_t count_a = Builders.build_aggregated_set(Iterators_Edge_a_d.head, Iterators_bag_1_a.head);
    (void)count_a;
    par::reducer<long> annotation_a(0, [&](long a, long b) { return a + b; });
    Builders.par_foreach_aggregate([&](const size_t tid, const uint32_t a_d) {
      TrieBuilder<long, MB>* Builder = Builders.builders.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_a_d = Iterators_Edge_a_d.iterators.at(tid);
      TrieIterator<long, MB>* Iterator_bag_1_a = Iterators_bag_1_a.iterators.at(tid);
      Iterator_Edge_a_d->get_next_block(0, a_d);
      const size_t count_d = Builder->build_aggregated_set(Iterator_Edge_a_d->get_block(1));
      const long intermediate_d = (long)1 * (count_d * 1);
      const long intermediate_a = (long)1 * Iterator_bag_1_a->get_annotation(0, a_d) * intermediate_d;
      annotation_a.update(tid, intermediate_a);
    });
    Builders.trie->annotation = annotation_a.evaluate(0);
    result = Builders.trie->annotation;
  }
  delete Trie_LollipopAgg_;
  return result;
}

/* BarbellAgg(;w) :- Edge(a,x) ⋈ bag_1(a;z) ⋈ bag_1(x;z)  (root bag, order [a,x];
 * the two triangle bags are deduplicated into one, IROptimizer.scala:64) */
static long bag_barbell_root(Trie<void*, MB>* Trie_Edge_0_1, Trie<long, MB>* Trie_bag_1, const std::string& out) {
  Trie<long, MB>* Trie_BarbellAgg_ = new Trie<long, MB>(out, 0, true);
  long result;
  {
    ParTrieBuilder<long, MB> Builders(Trie_BarbellAgg_, 2);
    ParTrieIterator<void*, MB> Iterators_Edge_a_x(Trie_Edge_0_1);
    ParTrieIterator<long, MB> Iterators_bag_1_a(Trie_bag_1);
    ParTrieIterator<long, MB> Iterators_bag_1_x(Trie_bag_1);
    const size_t count_a = Builders.build_aggregated_set(Iterators_Edge_a_x.head, Iterators_bag_1_a.head);
    (void)count_a;
    par::reducer<long> annotation_a(0, [&](long a, long b) { return a + b; });
    Builders.par_foreach_aggregate([&](const size_t tid, const uint32_t a_d) {
      TrieBuilder<long, MB>* Builder = Builders.builders.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_a_x = Iterators_Edge_a_x.iterators.at(tid);
      TrieIterator<long, MB>* Iterator_bag_1_a = Iterators_bag_1_a.iterators.at(tid);
      TrieIterator<long, MB>* Iterator_bag_1_x = Iterators_bag_1_x.iterators.at(tid);
      Iterator_Edge_a_x->get_next_block(0, a_d);
      const size_t count_x =
          Builder->build_aggregated_set(Iterator_Edge_a_x->get_block(1), Iterator_bag_1_x->get_block(0));
      (void)count_x;
      long annotation_x = (long)0;
      Builder->foreach_aggregate([&](const uint32_t x_d) {
        const long intermediate_x = (long)1 * Iterator_bag_1_x->get_annotation(0, x_d);
        annotation_x += intermediate_x;
      });
      const long intermediate_a = (long)1 * Iterator_bag_1_a->get_annotation(0, a_d) * annotation_x;
      annotation_a.update(tid, intermediate_a);
    });
    Builders.trie->annotation = annotation_a.evaluate(0);
    result = Builders.trie->annotation;
  }
  delete Trie_BarbellAgg_;
  return result;
}

/* ------------------------------------------------------- selection bags
 * A bag whose first attribute carries an equality selection and one
 * accessor is answered at the head (emitHeadContainsSelections,
 * EHGenerator.scala:681-701): get_next_block(selection) moves the
 * iterator's head to the selected value's child set, and the remaining
 * attribute is materialised with its annotation (SUM over the selected
 * attribute of 1, i.e. 1 per partner).
 *   bag_1_x_a_FliqueSelAgg(a;z) :- Edge(a,x), x=v   (order [x,a], trie Edge_1_0)
 *   bag_1_p_a_BarbellSelAgg(a;w) :- Edge(a,p), p=v  (order [p,a], trie Edge_1_0)
 *   bag_2_p_x_BarbellSelAgg(x;w) :- Edge(p,x), p=v  (order [p,x], trie Edge_0_1)
 * (QueryPlannerTest.scala:230-304).  Returns null when v heads no set: the
 * generated code would dereference a null block there.  A v above the
 * head's last value is treated the same way: on a dense head,
 * TrieBlock::get_next_block indexes the next-level array by value
 * (TrieBlock.hpp:88-95) and would read past its end. */
static Trie<long, MB>* bag_selected_partners(Trie<void*, MB>* Trie_Edge, uint32_t selection_0, const std::string& out) {
  mkdir(out.c_str(), 0755);
  mkdir((out + "/ram").c_str(), 0755);
  const Set<hybrid>* head_set = Trie_Edge->getHead()->get_const_set();
  if (head_set->cardinality == 0 || selection_0 > head_set->range) return nullptr;
  ParTrieIterator<void*, MB> Iterators_Edge(Trie_Edge);
  Iterators_Edge.get_next_block(selection_0);
  if (Iterators_Edge.head == nullptr) return nullptr;
  Trie<long, MB>* Trie_bag = new Trie<long, MB>(out, 1, true);
  {
    ParTrieBuilder<long, MB> Builders(Trie_bag, 2);
    const size_t count_a = Builders.build_set(Iterators_Edge.head);
    Builders.allocate_annotation();
    Builders.par_foreach_builder([&](const size_t tid, const uint32_t a_i, const uint32_t a_d) {
      TrieBuilder<long, MB>* Builder = Builders.builders.at(tid);
      Builder->set_annotation((long)1, a_i, a_d);
    });
    Builders.trie->num_rows = count_a;
  }
  return Trie_bag;
}

/* FliqueSelAgg(;z) root bag, order [a,b,c,d]: the FliqueAgg loop nest with
 * bag_1(a;z) joined at a (its head in a's intersection, z(a) multiplied in) */
static long bag_clique4_sel_root(Trie<void*, MB>* Trie_Edge_0_1, Trie<long, MB>* Trie_bag_1, const std::string& out) {
  typedef const TrieBlock<hybrid, MB>* TB;
  Trie<long, MB>* Trie_FliqueSelAgg_ = new Trie<long, MB>(out, 0, true);
  long result;
  {
    ParTrieBuilder<long, MB> Builders(Trie_FliqueSelAgg_, 4);
    ParTrieIterator<void*, MB> Iterators_Edge_c_d(Trie_Edge_0_1);
    ParTrieIterator<void*, MB> Iterators_Edge_b_c(Trie_Edge_0_1);
    ParTrieIterator<void*, MB> Iterators_Edge_b_d(Trie_Edge_0_1);
    ParTrieIterator<void*, MB> Iterators_Edge_a_c(Trie_Edge_0_1);
    ParTrieIterator<long, MB> Iterators_bag_1_a(Trie_bag_1);
    ParTrieIterator<void*, MB> Iterators_Edge_a_d(Trie_Edge_0_1);
    ParTrieIterator<void*, MB> Iterators_Edge_a_b(Trie_Edge_0_1);
    std::vector<TB> a_sets;
    a_sets.push_back(Iterators_Edge_a_c.head);
    a_sets.push_back(Iterators_bag_1_a.head);
    a_sets.push_back(Iterators_Edge_a_d.head);
    a_sets.push_back(Iterators_Edge_a_b.head);
    const size_t count_a = Builders.build_aggregated_set(&a_sets);
    (void)count_a;
    par::reducer<long> annotation_a(0, [&](long a, long b) { return a + b; });
    Builders.par_foreach_aggregate([&](const size_t tid, const uint32_t a_d) {
      TrieBuilder<long, MB>* Builder = Builders.builders.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_c_d = Iterators_Edge_c_d.iterators.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_b_c = Iterators_Edge_b_c.iterators.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_b_d = Iterators_Edge_b_d.iterators.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_a_c = Iterators_Edge_a_c.iterators.at(tid);
      TrieIterator<long, MB>* Iterator_bag_1_a = Iterators_bag_1_a.iterators.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_a_d = Iterators_Edge_a_d.iterators.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_a_b = Iterators_Edge_a_b.iterators.at(tid);
      Iterator_Edge_a_c->get_next_block(0, a_d);
      Iterator_Edge_a_d->get_next_block(0, a_d);
      Iterator_Edge_a_b->get_next_block(0, a_d);
      std::vector<TB> b_sets;
      b_sets.push_back(Iterator_Edge_b_c->get_block(0));
      b_sets.push_back(Iterator_Edge_b_d->get_block(0));
      b_sets.push_back(Iterator_Edge_a_b->get_block(1));
      const size_t count_b = Builder->build_aggregated_set(&b_sets);
      (void)count_b;
      long annotation_b = (long)0;
      Builder->foreach_aggregate([&](const uint32_t b_d) {
        Iterator_Edge_b_c->get_next_block(0, b_d);
        Iterator_Edge_b_d->get_next_block(0, b_d);
        std::vector<TB> c_sets;
        c_sets.push_back(Iterator_Edge_c_d->get_block(0));
        c_sets.push_back(Iterator_Edge_b_c->get_block(1));
        c_sets.push_back(Iterator_Edge_a_c->get_block(1));
        const size_t count_c = Builder->build_aggregated_set(&c_sets);
        (void)count_c;
        long annotation_c = (long)0;
        Builder->foreach_aggregate([&](const uint32_t c_d) {
          Iterator_Edge_c_d->get_next_block(0, c_d);
          std::vector<TB> d_sets;
          d_sets.push_back(Iterator_Edge_c_d->get_block(1));
          d_sets.push_back(Iterator_Edge_b_d->get_block(1));
          d_sets.push_back(Iterator_Edge_a_d->get_block(1));
          const size_t count_d = Builder->build_aggregated_set(&d_sets);
          const long intermediate_d = (long)1 * (count_d * 1);
          annotation_c += intermediate_d;
        });
        annotation_b += annotation_c;
      });
      const long intermediate_a = (long)1 * Iterator_bag_1_a->get_annotation(0, a_d) * annotation_b;
      annotation_a.update(tid, intermediate_a);
    });
    Builders.trie->annotation = annotation_a.evaluate(0);
    result = Builders.trie->annotation;
  }
  delete Trie_FliqueSelAgg_;
  return result;
}

/* bag_1_x_y_z_BarbellSelAgg(;w) :- Edge(y,z),Edge(x,z),Edge(x,y),bag_2(x;w)
 * (order [x,y,z]): a scalar, passed into the root bag */
static long bag_triangle_sel_scalar(Trie<void*, MB>* Trie_Edge_0_1, Trie<long, MB>* Trie_bag_2, const std::string& out) {
  typedef const TrieBlock<hybrid, MB>* TB;
  Trie<long, MB>* Trie_bag_xyz = new Trie<long, MB>(out, 0, true);
  long result;
  {
    ParTrieBuilder<long, MB> Builders(Trie_bag_xyz, 3);
    ParTrieIterator<void*, MB> Iterators_Edge_y_z(Trie_Edge_0_1);
    ParTrieIterator<void*, MB> Iterators_Edge_x_z(Trie_Edge_0_1);
    ParTrieIterator<void*, MB> Iterators_Edge_x_y(Trie_Edge_0_1);
    ParTrieIterator<long, MB> Iterators_bag_2_x(Trie_bag_2);
    std::vector<TB> x_sets;
    x_sets.push_back(Iterators_Edge_x_z.head);
    x_sets.push_back(Iterators_Edge_x_y.head);
    x_sets.push_back(Iterators_bag_2_x.head);
    const size_t count_x = Builders.build_aggregated_set(&x_sets);
    (void)count_x;
    par::reducer<long> annotation_x(0, [&](long a, long b) { return a + b; });
    Builders.par_foreach_aggregate([&](const size_t tid, const uint32_t x_d) {
      TrieBuilder<long, MB>* Builder = Builders.builders.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_y_z = Iterators_Edge_y_z.iterators.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_x_z = Iterators_Edge_x_z.iterators.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_x_y = Iterators_Edge_x_y.iterators.at(tid);
      TrieIterator<long, MB>* Iterator_bag_2_x = Iterators_bag_2_x.iterators.at(tid);
      Iterator_Edge_x_z->get_next_block(0, x_d);
      Iterator_Edge_x_y->get_next_block(0, x_d);
      const size_t count_y =
          Builder->build_aggregated_set(Iterator_Edge_y_z->get_block(0), Iterator_Edge_x_y->get_block(1));
      (void)count_y;
      long annotation_y = (long)0;
      Builder->foreach_aggregate([&](const uint32_t y_d) {
        Iterator_Edge_y_z->get_next_block(0, y_d);
        const size_t count_z =
            Builder->build_aggregated_set(Iterator_Edge_y_z->get_block(1), Iterator_Edge_x_z->get_block(1));
        const long intermediate_z = (long)1 * (count_z * 1);
        annotation_y += intermediate_z;
      });
      const long intermediate_x = (long)1 * Iterator_bag_2_x->get_annotation(0, x_d) * annotation_y;
      annotation_x.update(tid, intermediate_x);
    });
    Builders.trie->annotation = annotation_x.evaluate(0);
    result = Builders.trie->annotation;
  }
  delete Trie_bag_xyz;
  return result;
}

/* BarbellSelAgg(;w) root bag, order [a,b,c]: Edge(b,c), scalar bag,
 * bag_1_p_a(a;w), Edge(a,c), Edge(a,b) */
static long bag_barbell_sel_root(Trie<void*, MB>* Trie_Edge_0_1, Trie<long, MB>* Trie_bag_1, long scalar,
                                 const std::string& out) {
  typedef const TrieBlock<hybrid, MB>* TB;
  Trie<long, MB>* Trie_BarbellSelAgg_ = new Trie<long, MB>(out, 0, true);
  long result;
  {
    ParTrieBuilder<long, MB> Builders(Trie_BarbellSelAgg_, 3);
    ParTrieIterator<void*, MB> Iterators_Edge_b_c(Trie_Edge_0_1);
    ParTrieIterator<long, MB> Iterators_bag_1_a(Trie_bag_1);
    ParTrieIterator<void*, MB> Iterators_Edge_a_c(Trie_Edge_0_1);
    ParTrieIterator<void*, MB> Iterators_Edge_a_b(Trie_Edge_0_1);
    std::vector<TB> a_sets;
    a_sets.push_back(Iterators_bag_1_a.head);
    a_sets.push_back(Iterators_Edge_a_c.head);
    a_sets.push_back(Iterators_Edge_a_b.head);
    const size_t count_a = Builders.build_aggregated_set(&a_sets);
    (void)count_a;
    par::reducer<long> annotation_a(0, [&](long a, long b) { return a + b; });
    Builders.par_foreach_aggregate([&](const size_t tid, const uint32_t a_d) {
      TrieBuilder<long, MB>* Builder = Builders.builders.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_b_c = Iterators_Edge_b_c.iterators.at(tid);
      TrieIterator<long, MB>* Iterator_bag_1_a = Iterators_bag_1_a.iterators.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_a_c = Iterators_Edge_a_c.iterators.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_a_b = Iterators_Edge_a_b.iterators.at(tid);
      Iterator_Edge_a_c->get_next_block(0, a_d);
      Iterator_Edge_a_b->get_next_block(0, a_d);
      const size_t count_b =
          Builder->build_aggregated_set(Iterator_Edge_b_c->get_block(0), Iterator_Edge_a_b->get_block(1));
      (void)count_b;
      long annotation_b = (long)0;
      Builder->foreach_aggregate([&](const uint32_t b_d) {
        Iterator_Edge_b_c->get_next_block(0, b_d);
        const size_t count_c =
            Builder->build_aggregated_set(Iterator_Edge_b_c->get_block(1), Iterator_Edge_a_c->get_block(1));
        const long intermediate_c = (long)1 * (count_c * 1);
        annotation_b += intermediate_c;
      });
      const long intermediate_a = (long)1 * Iterator_bag_1_a->get_annotation(0, a_d) * annotation_b * scalar;
      annotation_a.update(tid, intermediate_a);
    });
    Builders.trie->annotation = annotation_a.evaluate(0);
    result = Builders.trie->annotation;
  }
  delete Trie_BarbellSelAgg_;
  return result;
}


/* PathAgg(;z) :- Edge(a,b),Edge(b,c),z:long<-[COUNT(*)].  Order [a,b,c];
 * c is read from one accessor, so its count is the set's cardinality
 * (TrieBuilder::build_aggregated_set of one block, TrieBuilder.cpp:223-240). */
static long bag_path2(Trie<void*, MB>* Trie_Edge_0_1, const std::string& out) {
  Trie<long, MB>* Trie_PathAgg_ = new Trie<long, MB>(out, 0, true);
  long result;
  {
    ParTrieBuilder<long, MB> Builders(Trie_PathAgg_, 3);
    ParTrieIterator<void*, MB> Iterators_Edge_a_b(Trie_Edge_0_1);
    ParTrieIterator<void*, MB> Iterators_Edge_b_c(Trie_Edge_0_1);
    const size_t count_a = Builders.build_aggregated_set(Iterators_Edge_a_b.head);
    (void)count_a;
    par::reducer<long> annotation_a(0, [&](long a, long b) { return a + b; });
    Builders.par_foreach_aggregate([&](const size_t tid, const uint32_t a_d) {
      TrieBuilder<long, MB>* Builder = Builders.builders.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_a_b = Iterators_Edge_a_b.iterators.at(tid);
      TrieIterator<void*, MB>* Iterator_Edge_b_c = Iterators_Edge_b_c.iterators.at(tid);
      Iterator_Edge_a_b->get_next_block(0, a_d);
      const size_t count_b =
          Builder->build_aggregated_set(Iterator_Edge_a_b->get_block(1), Iterator_Edge_b_c->get_block(0));
      (void)count_b;
      long annotation_b = (long)0;
      Builder->foreach_aggregate([&](const uint32_t b_d) {
        Iterator_Edge_b_c->get_next_block(0, b_d);
        const size_t count_c = Builder->build_aggregated_set(Iterator_Edge_b_c->get_block(1));
        const long intermediate_c = (long)1 * (count_c * 1);
        annotation_b += intermediate_c;
      });
      annotation_a.update(tid, annotation_b);
    });
    Builders.trie->annotation = annotation_a.evaluate(0);
    result = Builders.trie->annotation;
  }
  delete Trie_PathAgg_;
  return result;
}

#endif  // EH_GENERATED_BAGS_HPP
